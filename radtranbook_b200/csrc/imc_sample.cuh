// imc_sample.cuh — per-particle FP64 sampling of source positions and directions, shared
// by the single-problem and the batched source kernels (same code, same compile flags, so
// a batched instance draws exactly the particles its single-problem run draws).
#pragma once
#include <cmath>
#include <cuda_runtime.h>
#include "imc_device.cuh"

namespace imcsample {

using imcdev::G_SLAB;
using imcdev::G_SPHERE;
using imcdev::G_XY;
using imcdev::G_RZ;

__device__ __forceinline__ double pow4(double T) { const double t2 = T * T; return t2 * t2; }

// slab linear-T position in [0, dx], IMC/IMC1D.py:203-217
__device__ inline double slab_linear(double dx, double s, double T, double xi) {
  if (fabs(s) < 1e-6) return xi * dx;
  const double smax = 2.0 * T / (dx * dx);
  s = fmax(-smax, fmin(s, smax));
  const double q = s / (2.0 * T) - 1.0 / dx;
  const double disc = q * q + 2.0 * s * xi / (T * dx);
  return (-2.0 * T + s * dx + 2.0 * T * dx * sqrt(fmax(disc, 0.0))) / (2.0 * s);
}

// sphere linear-T^4 CDF inversion (bracketed Newton), IMC/IMC1D.py:578-626
__device__ inline double sphere_cdf(double r0, double r1, double a, double M, double xi) {
  const double C = a / 3.0 * (r1 * r1 * r1 - r0 * r0 * r0) + M / 4.0 * (pow4(r1) - pow4(r0));
  if (C <= 0.0) return r0 + xi * (r1 - r0);
  const double rhs = xi * C + (a / 3.0 * r0 * r0 * r0 + M / 4.0 * pow4(r0));
  double lo = r0, hi = r1, r = r0 + xi * (r1 - r0);
  for (int it = 0; it < 60; ++it) {
    const double r3 = r * r * r, r4 = r3 * r;
    const double g = a / 3.0 * r3 + M / 4.0 * r4 - rhs;
    if (fabs(g) < 1e-14 * (fabs(rhs) + 1e-30)) break;
    if (g < 0.0) lo = r; else hi = r;
    const double dg = r * r * (a + M * r);
    double rn = fabs(dg) > 1e-30 ? r - g / dg : 0.5 * (lo + hi);
    if (rn <= lo || rn >= hi) rn = 0.5 * (lo + hi);
    if (fabs(rn - r) < 1e-14 * (r1 - r0 + 1e-30)) { r = rn; break; }
    r = rn;
  }
  return r;
}

// cylinder linear-in-r CDF inversion (bracketed Newton), IMC/IMC2D.py:1293-1323
__device__ inline double rz_r_cdf(double r0, double r1, double a, double M, double xi) {
  const double C = a * 0.5 * (r1 * r1 - r0 * r0) + M / 3.0 * (r1 * r1 * r1 - r0 * r0 * r0);
  if (C <= 0.0) return sqrt(r0 * r0 + (r1 * r1 - r0 * r0) * xi);
  const double rhs = xi * C + a * 0.5 * r0 * r0 + M / 3.0 * r0 * r0 * r0;
  double lo = r0, hi = r1, r = sqrt(r0 * r0 + (r1 * r1 - r0 * r0) * xi);
  for (int it = 0; it < 50; ++it) {
    const double g = a * 0.5 * r * r + M / 3.0 * r * r * r - rhs;
    if (fabs(g) < 1e-14 * (fabs(rhs) + 1e-30)) break;
    if (g < 0.0) lo = r; else hi = r;
    const double dg = a * r + M * r * r;
    double rn = fabs(dg) > 1e-30 ? r - g / dg : 0.5 * (lo + hi);
    if (rn <= lo || rn >= hi) rn = 0.5 * (lo + hi);
    if (fabs(rn - r) < 1e-14 * (r1 - r0 + 1e-30)) { r = rn; break; }
    r = rn;
  }
  return r;
}

__device__ __forceinline__ void iso_dir(int geom, double ua, double ub, double& d1, double& d2) {
  if (geom == G_SLAB || geom == G_SPHERE) { d1 = 2.0 * ua - 1.0; d2 = 0.0; return; }
  if (geom == G_XY) {
    const double uz = 2.0 * ua - 1.0;
    const double rxy = sqrt(fmax(0.0, 1.0 - uz * uz));
    double sp, cp;
    sincospi(2.0 * ub, &sp, &cp);
    d1 = rxy * cp; d2 = rxy * sp;
  } else {
    d2 = 2.0 * ua - 1.0;      // eta
    d1 = cospi(2.0 * ub);     // mu_perp
  }
}

}  // namespace imcsample
