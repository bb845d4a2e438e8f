// speedy_ad.h -- reverse-mode automatic differentiation for one column, host and device.
//
// Adj<T> carries a value and the index of its node on a per-thread tape (TapeT<T>); every
// arithmetic operation on Adj values appends one node holding up to two parents and the local
// partial derivatives.  The reverse sweep walks the tape backwards once.  Ties of min/max split
// the derivative 0.5/0.5, as JAX's lax.min/lax.max JVP rules do; select (where) passes the
// derivative to the chosen branch only.  The tape arrays may be strided (stride = number of
// concurrent threads) so that threads of a warp touching the same node index coalesce.
#pragma once

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define SPD_HD __host__ __device__ __forceinline__
#else
#define SPD_HD inline
#endif

namespace spdad {

template <class T>
struct TapeT {
  int32_t* ia;
  int32_t* ib;
  T* pa;
  T* pb;
  T* adj;
  size_t stride;
  int n, cap;
  int overflow;

  SPD_HD int push(int a, T da, int b, T db) {
    if (a < 0 && b < 0) return -1;
    if (n >= cap) {
      overflow = 1;
      return -1;
    }
    const size_t o = (size_t)n * stride;
    ia[o] = a;
    pa[o] = da;
    ib[o] = b;
    pb[o] = db;
    adj[o] = T(0);
    return n++;
  }
  SPD_HD int leaf() {
    if (n >= cap) {
      overflow = 1;
      return -1;
    }
    const size_t o = (size_t)n * stride;
    ia[o] = -1;
    ib[o] = -1;
    pa[o] = T(0);
    pb[o] = T(0);
    adj[o] = T(0);
    return n++;
  }
  SPD_HD void seed(int i, T g) {
    if (i >= 0) adj[(size_t)i * stride] += g;
  }
  SPD_HD T grad(int i) const { return i >= 0 ? adj[(size_t)i * stride] : T(0); }
  SPD_HD void reverse() {
    for (int k = n - 1; k >= 0; --k) {
      const size_t o = (size_t)k * stride;
      const T g = adj[o];
      if (g == T(0)) continue;
      const int a = ia[o], b = ib[o];
      if (a >= 0) adj[(size_t)a * stride] += g * pa[o];
      if (b >= 0) adj[(size_t)b * stride] += g * pb[o];
    }
  }
};

template <class T>
struct Adj {
  T v;
  int i;
  TapeT<T>* t;
  SPD_HD Adj() : v(T(0)), i(-1), t(nullptr) {}
  SPD_HD Adj(T x) : v(x), i(-1), t(nullptr) {}
  SPD_HD Adj(T x, int idx, TapeT<T>* tp) : v(x), i(idx), t(tp) {}
};

template <class T>
SPD_HD TapeT<T>* tape_of(const Adj<T>& a, const Adj<T>& b) {
  return a.t ? a.t : b.t;
}

template <class T>
SPD_HD Adj<T> node(T v, const Adj<T>& a, T da, const Adj<T>& b, T db) {
  TapeT<T>* t = tape_of(a, b);
  if (!t) return Adj<T>(v);
  return Adj<T>(v, t->push(a.i, da, b.i, db), t);
}
template <class T>
SPD_HD Adj<T> node1(T v, const Adj<T>& a, T da) {
  if (!a.t) return Adj<T>(v);
  return Adj<T>(v, a.t->push(a.i, da, -1, T(0)), a.t);
}

template <class T> SPD_HD Adj<T> operator+(const Adj<T>& a, const Adj<T>& b) { return node(a.v + b.v, a, T(1), b, T(1)); }
template <class T> SPD_HD Adj<T> operator-(const Adj<T>& a, const Adj<T>& b) { return node(a.v - b.v, a, T(1), b, T(-1)); }
template <class T> SPD_HD Adj<T> operator*(const Adj<T>& a, const Adj<T>& b) { return node(a.v * b.v, a, b.v, b, a.v); }
template <class T> SPD_HD Adj<T> operator/(const Adj<T>& a, const Adj<T>& b) {
  const T r = a.v / b.v;
  return node(r, a, T(1) / b.v, b, -r / b.v);
}
template <class T> SPD_HD Adj<T> operator-(const Adj<T>& a) { return node1(-a.v, a, T(-1)); }

#define SPD_MIXED(OP)                                                                        \
  template <class T> SPD_HD Adj<T> operator OP(const Adj<T>& a, T b) { return a OP Adj<T>(b); } \
  template <class T> SPD_HD Adj<T> operator OP(T a, const Adj<T>& b) { return Adj<T>(a) OP b; }
SPD_MIXED(+)
SPD_MIXED(-)
SPD_MIXED(*)
SPD_MIXED(/)
#undef SPD_MIXED

template <class T> SPD_HD T val(const Adj<T>& a) { return a.v; }
SPD_HD float val(float a) { return a; }
SPD_HD double val(double a) { return a; }

template <class T> SPD_HD Adj<T> gexp(const Adj<T>& a) {
  const T e = exp(a.v);
  return node1(e, a, e);
}
template <class T> SPD_HD Adj<T> gsqrt(const Adj<T>& a) {
  const T s = sqrt(a.v);
  return node1(s, a, T(0.5) / s);
}
template <class T> SPD_HD Adj<T> gmax(const Adj<T>& a, const Adj<T>& b) {
  if (a.v > b.v) return node1(a.v, a, T(1));
  if (b.v > a.v) return node1(b.v, b, T(1));
  return node(a.v, a, T(0.5), b, T(0.5));
}
template <class T> SPD_HD Adj<T> gmin(const Adj<T>& a, const Adj<T>& b) {
  if (a.v < b.v) return node1(a.v, a, T(1));
  if (b.v < a.v) return node1(b.v, b, T(1));
  return node(a.v, a, T(0.5), b, T(0.5));
}
template <class T> SPD_HD Adj<T> gmax(const Adj<T>& a, T b) { return gmax(a, Adj<T>(b)); }
template <class T> SPD_HD Adj<T> gmax(T a, const Adj<T>& b) { return gmax(Adj<T>(a), b); }
template <class T> SPD_HD Adj<T> gmin(const Adj<T>& a, T b) { return gmin(a, Adj<T>(b)); }
template <class T> SPD_HD Adj<T> gmin(T a, const Adj<T>& b) { return gmin(Adj<T>(a), b); }

// plain scalars (the forward evaluation of the same code)
SPD_HD float gexp(float a) { return expf(a); }
SPD_HD double gexp(double a) { return exp(a); }
SPD_HD float gsqrt(float a) { return sqrtf(a); }
SPD_HD double gsqrt(double a) { return sqrt(a); }
SPD_HD float gmax(float a, float b) { return a > b ? a : (b > a ? b : a); }
SPD_HD double gmax(double a, double b) { return a > b ? a : (b > a ? b : a); }
SPD_HD float gmin(float a, float b) { return a < b ? a : (b < a ? b : a); }
SPD_HD double gmin(double a, double b) { return a < b ? a : (b < a ? b : a); }

template <class T> SPD_HD bool gisnan(const Adj<T>& a) { return a.v != a.v; }
SPD_HD bool gisnan(float a) { return a != a; }
SPD_HD bool gisnan(double a) { return a != a; }

}  // namespace spdad
