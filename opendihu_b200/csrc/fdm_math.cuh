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
