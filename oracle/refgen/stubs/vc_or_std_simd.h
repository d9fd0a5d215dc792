// Minimal stand-in for the Vc SIMD library (TEST INFRASTRUCTURE ONLY).  The reference's code generator
// writes its FastMonodomainSolver code against Vc::double_v; Vc itself is a third-party dependency that the
// reference downloads at build time and that is not available here.  This header provides the part of the
// Vc interface that the generator and the code it emits use, lane by lane in plain IEEE double arithmetic:
// a vector of W = 4 doubles (the AVX2 width, the reference's default), masks from comparisons, Vc::iif,
// Vc::where, and the elementary functions of <cmath> applied per lane (Vc's own vectorized exp/log differ
// from libm in the last bits; the cross-check compares the approximate-exponential variant, which uses none).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <iostream>
#include <vector>   // the real Vc headers bring these along; the emitted code relies on them

#ifndef HAVE_STDSIMD
#define HAVE_STDSIMD 1
#endif

namespace Vc {

constexpr int kLanes = 4;

struct VectorSpecialInitializerZero {};
struct VectorSpecialInitializerOne {};
constexpr VectorSpecialInitializerZero Zero{};
constexpr VectorSpecialInitializerOne One{};

struct double_m {
  bool v[kLanes];
  bool operator[](std::size_t i) const { return v[i]; }
  bool& operator[](std::size_t i) { return v[i]; }
};

inline double_m operator&&(const double_m& a, const double_m& b)
{
  double_m r;
  for (int i = 0; i < kLanes; i++)
    r.v[i] = a.v[i] && b.v[i];
  return r;
}
inline double_m operator||(const double_m& a, const double_m& b)
{
  double_m r;
  for (int i = 0; i < kLanes; i++)
    r.v[i] = a.v[i] || b.v[i];
  return r;
}
inline double_m operator!(const double_m& a)
{
  double_m r;
  for (int i = 0; i < kLanes; i++)
    r.v[i] = !a.v[i];
  return r;
}

struct double_v {
  double v[kLanes];
  double_v()
  {
    for (int i = 0; i < kLanes; i++)
      v[i] = 0.0;
  }
  double_v(double x)
  {
    for (int i = 0; i < kLanes; i++)
      v[i] = x;
  }
  double_v(VectorSpecialInitializerZero) : double_v(0.0) {}
  double_v(VectorSpecialInitializerOne) : double_v(1.0) {}
  static constexpr std::size_t size() { return kLanes; }
  double& operator[](std::size_t i) { return v[i]; }
  double operator[](std::size_t i) const { return v[i]; }
  template<class F>
  double_v apply(F f) const
  {
    double_v r;
    for (int i = 0; i < kLanes; i++)
      r.v[i] = f(v[i]);
    return r;
  }
  double_v& operator+=(const double_v& b)
  {
    for (int i = 0; i < kLanes; i++)
      v[i] += b.v[i];
    return *this;
  }
  double_v& operator-=(const double_v& b)
  {
    for (int i = 0; i < kLanes; i++)
      v[i] -= b.v[i];
    return *this;
  }
  double_v& operator*=(const double_v& b)
  {
    for (int i = 0; i < kLanes; i++)
      v[i] *= b.v[i];
    return *this;
  }
  double_v& operator/=(const double_v& b)
  {
    for (int i = 0; i < kLanes; i++)
      v[i] /= b.v[i];
    return *this;
  }
};

#define REFGEN_VC_BINARY(OP)                                                                \
  inline double_v operator OP(const double_v& a, const double_v& b)                         \
  {                                                                                         \
    double_v r;                                                                             \
    for (int i = 0; i < kLanes; i++)                                                        \
      r.v[i] = a.v[i] OP b.v[i];                                                            \
    return r;                                                                               \
  }                                                                                         \
  inline double_v operator OP(double a, const double_v& b) { return double_v(a) OP b; }     \
  inline double_v operator OP(const double_v& a, double b) { return a OP double_v(b); }
REFGEN_VC_BINARY(+)
REFGEN_VC_BINARY(-)
REFGEN_VC_BINARY(*)
REFGEN_VC_BINARY(/)
#undef REFGEN_VC_BINARY

inline double_v operator-(const double_v& a)
{
  double_v r;
  for (int i = 0; i < kLanes; i++)
    r.v[i] = -a.v[i];
  return r;
}
inline double_v operator+(const double_v& a) { return a; }

#define REFGEN_VC_COMPARE(OP)                                                               \
  inline double_m operator OP(const double_v& a, const double_v& b)                         \
  {                                                                                         \
    double_m r;                                                                             \
    for (int i = 0; i < kLanes; i++)                                                        \
      r.v[i] = a.v[i] OP b.v[i];                                                            \
    return r;                                                                               \
  }                                                                                         \
  inline double_m operator OP(double a, const double_v& b) { return double_v(a) OP b; }     \
  inline double_m operator OP(const double_v& a, double b) { return a OP double_v(b); }
REFGEN_VC_COMPARE(<)
REFGEN_VC_COMPARE(<=)
REFGEN_VC_COMPARE(>)
REFGEN_VC_COMPARE(>=)
REFGEN_VC_COMPARE(==)
REFGEN_VC_COMPARE(!=)
#undef REFGEN_VC_COMPARE

inline double_v iif(const double_m& m, const double_v& a, const double_v& b)
{
  double_v r;
  for (int i = 0; i < kLanes; i++)
    r.v[i] = m.v[i] ? a.v[i] : b.v[i];
  return r;
}
inline double_v iif(bool m, const double_v& a, const double_v& b) { return m ? a : b; }

struct WhereProxy {
  double_m m;
  double_v& x;
  WhereProxy& operator=(const double_v& y)
  {
    for (int i = 0; i < kLanes; i++)
      if (m.v[i])
        x.v[i] = y.v[i];
    return *this;
  }
  WhereProxy& operator+=(const double_v& y)
  {
    for (int i = 0; i < kLanes; i++)
      if (m.v[i])
        x.v[i] += y.v[i];
    return *this;
  }
};
inline WhereProxy where(const double_m& m, double_v& x) { return WhereProxy{m, x}; }

inline bool any_of(const double_m& m)
{
  for (int i = 0; i < kLanes; i++)
    if (m.v[i])
      return true;
  return false;
}
inline bool all_of(const double_m& m)
{
  for (int i = 0; i < kLanes; i++)
    if (!m.v[i])
      return false;
  return true;
}
inline bool none_of(const double_m& m) { return !any_of(m); }

#define REFGEN_VC_UNARY(NAME, FN)                                                           \
  inline double_v NAME(const double_v& a)                                                   \
  {                                                                                         \
    double_v r;                                                                             \
    for (int i = 0; i < kLanes; i++)                                                        \
      r.v[i] = FN(a.v[i]);                                                                  \
    return r;                                                                               \
  }
REFGEN_VC_UNARY(exp, std::exp)
REFGEN_VC_UNARY(log, std::log)
REFGEN_VC_UNARY(abs, std::fabs)
REFGEN_VC_UNARY(fabs, std::fabs)
REFGEN_VC_UNARY(sqrt, std::sqrt)
REFGEN_VC_UNARY(floor, std::floor)
REFGEN_VC_UNARY(ceil, std::ceil)
#undef REFGEN_VC_UNARY

inline double_m isfinite(const double_v& a)
{
  double_m r;
  for (int i = 0; i < kLanes; i++)
    r.v[i] = std::isfinite(a.v[i]);
  return r;
}

} // namespace Vc
