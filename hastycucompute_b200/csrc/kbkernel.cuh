// Kaiser-Bessel spreading kernel: parameters, a piecewise-polynomial device evaluator fitted
// on the host, and the analytic deapodisation factors.
//
// phi(z) = I0(beta * sqrt(1 - (2z/w)^2)) / I0(beta) for |z| < w/2 (fine-grid units).
// A point at fine coordinate u touches the w cells l = i0 .. i0+w-1 with i0 = ceil(u - w/2);
// with t = i0 - (u - w/2) in [0,1), tap d sees z = d - w/2 + t. Each tap d has its own
// polynomial P_d(s), s = 2t - 1, fitted at Chebyshev nodes, so the device evaluates the kernel
// by Horner's rule instead of a Bessel function.
#pragma once

#include <stdint.h>

namespace hb {

constexpr int kMaxWidth = 16;
constexpr int kMaxDeg = 15;

struct KbPoly {
    int w;      // taps per non-unit axis
    int deg;    // polynomial degree
    float hw;   // w / 2
    float coef[kMaxWidth][kMaxDeg + 1];  // P_d(s) = sum_m coef[d][m] s^m
};

// Host: beta for width w and upsampling factor sigma (Beatty et al., IEEE TMI 2005).
double kb_beta(int w, double sigma);
// Host: I0 by its power series, double precision.
double bessel_i0(double x);
// Host: phi(z), double precision.
double kb_phi(double z, int w, double beta);
// Host: Fourier transform of phi at xi cycles per grid unit, int phi(z) exp(-2 pi i xi z) dz.
double kb_phihat(double xi, int w, double beta);
// Host: fits the per-tap polynomials; returns the max abs error seen on a dense check grid.
double kb_fit(KbPoly* p, int w, double beta);

#ifdef __CUDACC__
// Device: evaluates the w taps of a point with fractional offset t in [0,1).
// `coef` points at a shared-memory copy of KbPoly::coef (row stride kMaxDeg+1).
__device__ __forceinline__ float kb_tap(const float* coef, int deg, int d, float s) {
    const float* c = coef + d * (kMaxDeg + 1);
    float acc = c[deg];
    for (int m = deg - 1; m >= 0; --m) acc = fmaf(acc, s, c[m]);
    return acc;
}
// Device: d phi / dz for tap d (= 2 dP/ds, since z = d - w/2 + (s+1)/2).
__device__ __forceinline__ float kb_tap_deriv(const float* coef, int deg, int d, float s) {
    const float* c = coef + d * (kMaxDeg + 1);
    float acc = (float)deg * c[deg];
    for (int m = deg - 1; m >= 1; --m) acc = fmaf(acc, s, (float)m * c[m]);
    return 2.f * acc;
}
#endif

}  // namespace hb
