/* Math helpers of the CPU oracle.  TEST INFRASTRUCTURE ONLY: nothing in the product links this.
 *
 * oracle_approx_exp / oracle_approx_log restate the helpers the reference emits when
 * "approximateExponentialFunction" is true (core/src/cellml/source_code_generator/
 * 03_generator_vc.cpp:385-407 and :436-490):
 *   exp(x) ~ (1 + x/1024)^1024, evaluated as ten successive squarings;
 *   log(x) ~ a 4th/6th order Taylor polynomial of log around 1, 3 or 9 (chosen by the range of x),
 *            followed by one Newton step y -= 1 - x/exp~(y) against the approximate exp.
 * The Taylor coefficients are the plain series coefficients log(a) + t/a - t^2/(2a^2) + t^3/(3a^3) - t^4/(4a^4)
 * (plus the t^5, t^6 terms around 1); the summation order matches the reference so that the
 * oracle reproduces its rounding.
 */
#pragma once
#include <math.h>

static inline double oracle_approx_exp(double x)
{
  double y = 1.0 + x / 1024.;
  for (int i = 0; i < 10; i++)
    y *= y;
  return y;
}

static inline double oracle_approx_log(double x)
{
  const double t1 = x - 1;
  const double t1_2 = t1 * t1;
  const double t1_4 = t1_2 * t1_2;
  const double t1_6 = t1_4 * t1_2;
  const double r1 = t1 - 0.5 * t1_2 + 1. / 3 * t1_2 * t1 - 0.25 * t1_4 + 0.2 * t1_4 * t1 - 1. / 6 * t1_6;

  const double t3 = x - 3;
  const double t3_2 = t3 * t3;
  const double t3_4 = t3_2 * t3_2;
  /* log(3), 1/3, 1/18, 1/81, 1/324 */
  const double r3 = 1.0986122886681098 + 1. / 3 * t3 - 0.05555555555555555 * t3_2 + 0.012345679012345678 * t3_2 * t3
                    - 0.0030864197530864196 * t3_4;

  const double t9 = x - 9;
  const double t9_2 = t9 * t9;
  const double t9_4 = t9_2 * t9_2;
  /* log(9), 1/9, 1/162, 1/2187, 1/26244 */
  const double r9 = 2.1972245773362196 + 1. / 9 * t9 - 0.006172839506172839 * t9_2 + 0.0004572473708276177 * t9_2 * t9
                    - 3.8103947568968146e-05 * t9_4;

  double r = r1;
  if (x >= 2 && x < 6)
    r = r3;
  else if (x >= 6)
    r = r9;
  r -= (1 - x / oracle_approx_exp(r));
  return r;
}
