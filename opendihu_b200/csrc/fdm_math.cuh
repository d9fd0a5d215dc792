// Math policies for the generated CellML right-hand sides.
//
// fdm_math_exact:  exp/log as the model file writes them.  FP64 uses the CUDA double-precision
//                  functions; FP32 uses the SFU (ex2/lg2) intrinsics, the FP32-reaction mode's
//                  precision contract being "Vm within 0.1 mV of the FP64 oracle".
// fdm_math_approx: the reference's "approximateExponentialFunction" helpers
//                  (core/src/cellml/source_code_generator/03_generator_vc.cpp:385-407, :436-490):
//                  exp(x) ~ (1 + x/1024)^1024 and a piecewise Taylor log refined by one Newton step.
//                  In FP64 the squaring chain is evaluated literally, giving the reference's rounding.
//                  In FP32 ten squarings would amplify the rounding of 1 + x/1024 by 1024, so the
//                  same function is evaluated as exp(1024*log1p(x/1024)), with log1p from its power
//                  series (alternating terms (-1)^(k+1) s^k / k, s = x/1024) and the SFU exponential;
//                  arguments beyond the series' range fall back to the FP64 squaring chain.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

// single SFU instructions for the FP32 form of the right-hand sides (relative error ~2^-22):
// 2^x, 1/x and log2(x), flushing denormals (the FP32 reaction is compiled with -ftz=true)
__device__ __forceinline__ float fdm_ex2(float x)
{
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float fdm_rcp(float x)
{
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float fdm_lg2(float x)
{
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// --------------------------------------------------------------------------------------------
// fdm_f2: two FP32 values (two nodes) evaluated by one packed sm_100 instruction (FADD2 / FMUL2 /
// FFMA2 through __fadd2_rn / __fmul2_rn / __ffma2_rn).  The generated paired right-hand side
// (rates_fast2) is the FP32 form written over this type, so one instruction stream advances two
// nodes.  A product is kept unevaluated (fdm_f2_prod) until it meets an addend, so a*b + c becomes
// one FFMA2 as a scalar a*b + c becomes one FFMA.  Transcendentals (ex2, rcp, lg2) have no packed
// form and run per component.
// --------------------------------------------------------------------------------------------
struct fdm_f2 {
  float2 v;
  __device__ __forceinline__ fdm_f2() {}
  __device__ __forceinline__ explicit fdm_f2(double c) : v(make_float2((float)c, (float)c)) {}
  __device__ __forceinline__ explicit fdm_f2(float c) : v(make_float2(c, c)) {}
  __device__ __forceinline__ fdm_f2(float a, float b) : v(make_float2(a, b)) {}
  __device__ __forceinline__ fdm_f2(float2 x) : v(x) {}
};
struct fdm_f2_prod {
  float2 a, b;
  __device__ __forceinline__ operator fdm_f2() const { return fdm_f2(__fmul2_rn(a, b)); }
};
struct fdm_b2 {
  bool x, y;
};

// a - b as one packed subtraction (PTX sub.f32x2; there is no packed-subtract intrinsic)
__device__ __forceinline__ float2 fdm_sub2(float2 a, float2 b)
{
  unsigned long long ra, rb, rd;
  memcpy(&ra, &a, 8);
  memcpy(&rb, &b, 8);
  asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
  float2 d;
  memcpy(&d, &rd, 8);
  return d;
}
// -a: one packed subtraction from zero (two scalar negations would cost two instructions)
__device__ __forceinline__ float2 fdm_neg2(float2 a) { return fdm_sub2(make_float2(0.f, 0.f), a); }
__device__ __forceinline__ fdm_f2 operator-(fdm_f2 a) { return fdm_f2(fdm_neg2(a.v)); }
__device__ __forceinline__ fdm_f2 operator+(fdm_f2 a) { return a; }
__device__ __forceinline__ fdm_f2_prod operator-(fdm_f2_prod p) { return fdm_f2_prod{fdm_neg2(p.a), p.b}; }
__device__ __forceinline__ fdm_f2_prod operator*(fdm_f2 a, fdm_f2 b) { return fdm_f2_prod{a.v, b.v}; }
__device__ __forceinline__ fdm_f2 operator+(fdm_f2 a, fdm_f2 b) { return fdm_f2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ fdm_f2 operator-(fdm_f2 a, fdm_f2 b) { return fdm_f2(fdm_sub2(a.v, b.v)); }
__device__ __forceinline__ fdm_f2 operator+(fdm_f2_prod p, fdm_f2 c) { return fdm_f2(__ffma2_rn(p.a, p.b, c.v)); }
__device__ __forceinline__ fdm_f2 operator+(fdm_f2 c, fdm_f2_prod p) { return fdm_f2(__ffma2_rn(p.a, p.b, c.v)); }
// a b - c and c - a b: a product and a packed subtraction (the negated operand of a fused form would
// cost a separate instruction as well); the generator writes constant subtrahends as negative addends
__device__ __forceinline__ fdm_f2 operator-(fdm_f2_prod p, fdm_f2 c) { return fdm_f2(fdm_sub2(__fmul2_rn(p.a, p.b), c.v)); }
__device__ __forceinline__ fdm_f2 operator-(fdm_f2 c, fdm_f2_prod p) { return fdm_f2(fdm_sub2(c.v, __fmul2_rn(p.a, p.b))); }
__device__ __forceinline__ fdm_f2 operator+(fdm_f2_prod p, fdm_f2_prod q) { return p + fdm_f2(q); }
__device__ __forceinline__ fdm_f2 operator-(fdm_f2_prod p, fdm_f2_prod q) { return p - fdm_f2(q); }
__device__ __forceinline__ fdm_f2& operator+=(fdm_f2& a, fdm_f2 b) { return a = a + b; }
__device__ __forceinline__ fdm_f2& operator+=(fdm_f2& a, fdm_f2_prod p) { return a = p + a; }
__device__ __forceinline__ fdm_f2 fdm_ex2(fdm_f2 x) { return fdm_f2(fdm_ex2(x.v.x), fdm_ex2(x.v.y)); }
__device__ __forceinline__ fdm_f2 fdm_rcp(fdm_f2 x) { return fdm_f2(fdm_rcp(x.v.x), fdm_rcp(x.v.y)); }
__device__ __forceinline__ fdm_f2 fdm_lg2(fdm_f2 x) { return fdm_f2(fdm_lg2(x.v.x), fdm_lg2(x.v.y)); }
__device__ __forceinline__ fdm_f2 operator/(fdm_f2 a, fdm_f2 b) { return a * fdm_rcp(b); }
__device__ __forceinline__ fdm_f2 fabs(fdm_f2 x) { return fdm_f2(fabsf(x.v.x), fabsf(x.v.y)); }
__device__ __forceinline__ fdm_f2 sqrt(fdm_f2 x) { return fdm_f2(sqrtf(x.v.x), sqrtf(x.v.y)); }
__device__ __forceinline__ fdm_f2 fdm_powf_pair(fdm_f2 x, fdm_f2 y)
{
  return fdm_f2(__powf(x.v.x, y.v.x), __powf(x.v.y, y.v.y));
}
#define FDM_F2_CMP(op)                                                                                   \
  __device__ __forceinline__ fdm_b2 operator op(fdm_f2 a, fdm_f2 b) { return fdm_b2{a.v.x op b.v.x, a.v.y op b.v.y}; }
FDM_F2_CMP(<)
FDM_F2_CMP(<=)
FDM_F2_CMP(>)
FDM_F2_CMP(>=)
FDM_F2_CMP(==)
FDM_F2_CMP(!=)
#undef FDM_F2_CMP
__device__ __forceinline__ fdm_b2 operator&&(fdm_b2 a, fdm_b2 b) { return fdm_b2{a.x && b.x, a.y && b.y}; }
__device__ __forceinline__ fdm_b2 operator||(fdm_b2 a, fdm_b2 b) { return fdm_b2{a.x || b.x, a.y || b.y}; }
__device__ __forceinline__ fdm_b2 operator!(fdm_b2 a) { return fdm_b2{!a.x, !a.y}; }
// per-component select (the paired form of c ? a : b; both operands are evaluated)
__device__ __forceinline__ fdm_f2 fdm_sel(fdm_b2 c, fdm_f2 a, fdm_f2 b)
{
  return fdm_f2(c.x ? a.v.x : b.v.x, c.y ? a.v.y : b.v.y);
}

// --------------------------------------------------------------------------------------------
// Batched reciprocals (simultaneous inversion): with q = d0 d1 [d2] one SFU reciprocal gives
// 1/d_k = (1/q) * (product of the other factors), three multiplications per saved reciprocal.
// Valid while q stays inside the FP32 range: for the Hodgkin-Huxley denominators
// exp(-(Vm+k)/10) c -/+ 1 that holds for Vm > -340 mV.  Outside it q is inf or 0 and the
// reciprocals become NaN, which the solver's non-finite check reports (FDM_ERR_NAN); the
// FP32-reaction mode is specified for physiological potentials.  No range test is made: a
// branch inside the right-hand side costs more than the reciprocals it saves.
// --------------------------------------------------------------------------------------------
// 1 - 2^t without cancellation and never exactly 0, for the FP32 form of 1 - exp(u) (t = u log2 e): for
// |t| < 2^-6 the series -x (1 + x/2 + x^2/6), x = t ln 2 (relative error below 2^-26 there), else 1 - ex2(t);
// t = 0 gives the smallest normal float instead of 0, so a removable singularity x / (1 - e^-ax) at x = 0
// evaluates to 0 rather than 0/0
__device__ __forceinline__ float fdm_1mexp2(float t)
{
  const float x = t * 0.69314718055994531f;
  const float series = -x * (1.f + x * (0.5f + x * (1.f / 6.f)));
  float d = fabsf(t) < 0.015625f ? series : 1.f - fdm_ex2(t);
  return d == 0.f ? 1.17549435e-38f : d;
}
__device__ __forceinline__ fdm_f2 fdm_1mexp2(fdm_f2 t) { return fdm_f2(fdm_1mexp2(t.v.x), fdm_1mexp2(t.v.y)); }
__device__ __forceinline__ double fdm_1mexp2(double t)
{
  const double d = -expm1(t * 0.69314718055994531);
  return d == 0.0 ? 2.2250738585072014e-308 : d;
}

template<class R>
__device__ __forceinline__ void fdm_rcp_batch(R d0, R d1, R& r0, R& r1)
{
  const R iv = fdm_rcp(R(d0 * d1));
  r0 = iv * d1;
  r1 = iv * d0;
}

template<class R>
__device__ __forceinline__ void fdm_rcp_batch(R d0, R d1, R d2, R& r0, R& r1, R& r2)
{
  const R q1 = d0 * d1;
  const R iv = fdm_rcp(R(q1 * d2));
  r2 = iv * q1;
  const R t = iv * d2; // 1/(d0 d1)
  r0 = t * d1;
  r1 = t * d0;
}

struct fdm_math_exact {
  // derivatives for the adjoint: d exp(x)/dx = exp(x), d log(x)/dx = 1/x
  template<class R>
  __device__ __forceinline__ static R dexp(R x, R ex) { (void)x; return ex; }
  template<class R>
  __device__ __forceinline__ static R dlog(R x, R lx) { (void)lx; return (R)1 / x; }
  __device__ __forceinline__ static double exp(double x) { return ::exp(x); }
  __device__ __forceinline__ static float exp(float x) { return __expf(x); }
  __device__ __forceinline__ static double log(double x) { return ::log(x); }
  __device__ __forceinline__ static float log(float x) { return __logf(x); }
  __device__ __forceinline__ static double pow(double x, double y) { return ::pow(x, y); }
  __device__ __forceinline__ static float pow(float x, float y) { return __powf(x, y); }
};

__device__ __forceinline__ double fdm_approx_exp_d(double x)
{
  double y = 1.0 + x / 1024.;
#pragma unroll
  for (int i = 0; i < 10; i++)
    y *= y;
  return y;
}

__device__ __forceinline__ float fdm_approx_exp_f(float x)
{
  // 1024*log1p(x/1024) = x - x^2/2048 + x^3/(3*1024^2) - x^4/(4*1024^3) + ...; the truncation
  // after the x^7 term is below 3e-9 for |x| <= 40.
  if (fabsf(x) > 40.f)
    return (float)fdm_approx_exp_d((double)x);
  const float c2 = -1.f / 2048.f;
  const float c3 = 1.f / (3.f * 1048576.f);
  const float c4 = -1.f / (4.f * 1073741824.f);
  const float c5 = 1.f / (5.f * 1099511627776.f);
  const float c6 = -1.f / (6.f * 1125899906842624.f);
  const float c7 = 1.f / (7.f * 1152921504606846976.f);
  float p = fmaf(x, c7, c6);
  p = fmaf(x, p, c5);
  p = fmaf(x, p, c4);
  p = fmaf(x, p, c3);
  p = fmaf(x, p, c2);
  p = fmaf(x, p, 1.f);
  return __expf(x * p);
}

template<class R>
__device__ __forceinline__ R fdm_approx_log_poly(R x)
{
  const R t1 = x - R(1);
  const R t1_2 = t1 * t1;
  const R t1_4 = t1_2 * t1_2;
  const R t1_6 = t1_4 * t1_2;
  const R r1 = t1 - R(0.5) * t1_2 + R(1. / 3) * t1_2 * t1 - R(0.25) * t1_4 + R(0.2) * t1_4 * t1 - R(1. / 6) * t1_6;
  const R t3 = x - R(3);
  const R t3_2 = t3 * t3;
  const R t3_4 = t3_2 * t3_2;
  const R r3 = R(1.0986122886681098) + R(1. / 3) * t3 - R(0.05555555555555555) * t3_2
               + R(0.012345679012345678) * t3_2 * t3 - R(0.0030864197530864196) * t3_4;
  const R t9 = x - R(9);
  const R t9_2 = t9 * t9;
  const R t9_4 = t9_2 * t9_2;
  const R r9 = R(2.1972245773362196) + R(1. / 9) * t9 - R(0.006172839506172839) * t9_2
               + R(0.0004572473708276177) * t9_2 * t9 - R(3.8103947568968146e-05) * t9_4;
  R r = r1;
  if (x >= R(2) && x < R(6))
    r = r3;
  else if (x >= R(6))
    r = r9;
  return r;
}

struct fdm_math_approx {
  // d/dx (1 + x/1024)^1024 = (1 + x/1024)^1023; the log approximation is differentiated as 1/x
  template<class R>
  __device__ __forceinline__ static R dexp(R x, R ex) { return ex / ((R)1 + x / (R)1024); }
  template<class R>
  __device__ __forceinline__ static R dlog(R x, R lx) { (void)lx; return (R)1 / x; }
  __device__ __forceinline__ static double exp(double x) { return fdm_approx_exp_d(x); }
  __device__ __forceinline__ static float exp(float x) { return fdm_approx_exp_f(x); }
  __device__ __forceinline__ static double log(double x)
  {
    double r = fdm_approx_log_poly<double>(x);
    r -= (1 - x / fdm_approx_exp_d(r));
    return r;
  }
  __device__ __forceinline__ static float log(float x)
  {
    float r = fdm_approx_log_poly<float>(x);
    r -= (1.f - __fdividef(x, fdm_approx_exp_f(r)));
    return r;
  }
  __device__ __forceinline__ static double pow(double x, double y) { return ::pow(x, y); }
  __device__ __forceinline__ static float pow(float x, float y) { return __powf(x, y); }
};
