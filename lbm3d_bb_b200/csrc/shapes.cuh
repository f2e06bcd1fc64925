// shapes.cuh — the reference's planar body shapes in FP32: the NACA 4-digit band
// (solid flags) and the level-set functions phi of the interpolated bounce-back.
//
// Include only from translation units compiled with --fmad=false: every expression
// rounds as written, exactly like the CPU restatement built with -ffp-contract=off.
#pragma once
#include "lbm_internal.cuh"

namespace lbm {

// NACA 4-digit band (Geometry.jl:325-356); cos(atan(s)) as 1/sqrt(1+s^2), x^4 as
// (x*x)*(x*x) — both sides of the parity check use this form.
__device__ __forceinline__ void naca_upper_lower(float x, float c, float m, float p, float t, float x_int, float* yL,
                                 float* yU) {
  const float xbar = x / c;
  const float xbi = fmaxf(0.0f, x_int * xbar);
  const float rt = sqrtf(xbi);
  const float x2 = xbi * xbi;
  const float x3 = x2 * xbi;
  const float x4 = x2 * x2;
  const float yt = 5.0f * t * c * (0.2969f * rt - 0.1260f * xbi - 0.3516f * x2 + 0.2843f * x3 - 0.1015f * x4);
  float yc, dycb;
  if (m == 0.0f || p == 0.0f) {
    yc = 0.0f;
    dycb = 0.0f;
  } else if (xbar < p) {
    yc = m / (p * p) * (2.0f * p * xbar - xbar * xbar);
    dycb = 2.0f * m / (p * p) * (p - xbar);
  } else {
    const float den = 1.0f - p;
    const float den2 = den * den;
    yc = m / den2 * ((1.0f - 2.0f * p) + 2.0f * p * xbar - xbar * xbar);
    dycb = 2.0f * m / den2 * (p - xbar);
  }
  const float s = dycb / c;
  const float czv = 1.0f / sqrtf(1.0f + s * s);
  *yU = yc + yt * czv;
  *yL = yc - yt * czv;
}

// phi_cylinder_lat (Geometry.jl:365-369): signed distance to the circle.
__device__ __forceinline__ float phi_cylinder(float x, float y, float xc, float yc, float R) {
  const float dx = x - xc, dy = y - yc;
  return sqrtf(dx * dx + dy * dy) - R;
}

// phi_airfoil_lat (Geometry.jl:372-392): quasi signed distance to the NACA band, negative
// inside; hypot(a, b) evaluated as sqrt(a*a + b*b) (so that CPU and GPU round alike).
__device__ __forceinline__ float phi_airfoil(float xw, float yw, float xc, float yc, float ct, float st,
                                             float chord, float m, float p, float t, float x_int,
                                             float x_le_offset) {
  const float dx = xw - xc, dy = yw - yc;
  const float xB = ct * dx + st * dy;
  const float yB = -st * dx + ct * dy;
  const float xle = xB + x_le_offset;
  if (xle < 0.0f) return sqrtf(xle * xle + yB * yB);
  if (xle > chord) {
    const float a = xle - chord;
    return sqrtf(a * a + yB * yB);
  }
  float yL, yU;
  naca_upper_lower(xle, chord, m, p, t, x_int, &yL, &yU);
  if ((yB >= yL) && (yB <= yU)) return -fminf(yU - yB, yB - yL);
  return (yB > yU) ? (yB - yU) : (yL - yB);
}

}  // namespace lbm
