// WENO7 face reconstruction shared by the stage kernels.
#pragma once

#include "common.cuh"

namespace cosenu {

// WENO7 face value from the 7-point stencil a..g = u[-3..3] about the cell
// whose right face (j+1/2) is reconstructed with left-biased weights
// (rflux of src/rhs_fv.hpp:37-71).  Smoothness indicators and candidate
// polynomials of the four 4-point sub-stencils; nonlinear weights
// gamma_r / (eps + beta_r)^2 with gamma = (4, 18, 12, 1)/35 and eps = 1e-6.
// FP64: the indicators and the candidate values are evaluated on differences
// from the centre value d (the indicators are invariant under a constant
// shift and each candidate's weights sum to 12, so the face is d plus the
// weighted differences: 15 fewer FP64 operations per face and less
// cancellation), and the four weights are brought to a common denominator,
// so that the face is d + num / den.  gamma and the 12 ride on the
// candidates' coefficients (gamma_r / 12 x the integer weights) and gamma on
// den, not on the weights; den = 4 w0 + 18 w1 + 12 w2 + w3 is three FMAs.
__device__ __forceinline__ void weno7_parts(double a, double b, double c, double d, double e,
                                            double f, double g, double &num, double &den)
{
    const double eps = 1e-6;
    const double A = a - d, B = b - d, Cc = c - d, E = e - d, F = f - d, G = g - d;
    double s0 = E * (11003. * E - 17246. * F + 4642. * G) + F * (7043. * F - 3882. * G) +
                547. * G * G;
    double s1 = Cc * (547. * Cc + 1922. * E - 494. * F) + E * (2843. * E - 1642. * F) +
                267. * F * F;
    double s2 = B * (267. * B - 1642. * Cc - 494. * E) + Cc * (2843. * Cc + 1922. * E) +
                547. * E * E;
    double s3 = A * (547. * A - 3882. * B + 4642. * Cc) + B * (7043. * B - 17246. * Cc) +
                11003. * Cc * Cc;
    // gamma_r x (candidate value - d): 12 x (candidate - d) has integer
    // weights summing to 12, scaled here by gamma_r / 12 = 1/3, 3/2, 1, 1/12
    double q0 = (13. / 3.) * E - (5. / 3.) * F + (1. / 3.) * G;
    double q1 = -1.5 * Cc + 10.5 * E - 1.5 * F;
    double q2 = B - 5. * Cc + 3. * E;
    double q3 = -0.25 * A + (13. / 12.) * B - (23. / 12.) * Cc;
    double d0 = (eps + s0) * (eps + s0);
    double d1 = (eps + s1) * (eps + s1);
    double d2 = (eps + s2) * (eps + s2);
    double d3 = (eps + s3) * (eps + s3);
    double d01 = d0 * d1, d23 = d2 * d3;
    // the weights without gamma: w_r = prod_{k != r} d_k
    double w0 = d1 * d23, w1 = d0 * d23, w2 = d01 * d3, w3 = d01 * d2;
    num = w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3;
    den = w3 + 4. * w0 + 18. * w1 + 12. * w2;
}

__device__ __forceinline__ double weno7_face(double a, double b, double c, double d, double e,
                                             double f, double g)
{
    double num, den;
    weno7_parts(a, b, c, d, e, f, g, num, den);
    return d + num / den;
}

// 1 / D0 .. 1 / D3 from one division: the product of the four, its
// reciprocal, then products of the others.  Denominators of weno7_parts lie
// in [3e-35, 2e33] where the stencil differences are at most 2 in magnitude
// (density-matrix entries of O(1)), so the product of four stays far inside
// the FP64 range.  Explicit round-to-nearest operations: the same
// inputs give the same bits wherever this is evaluated (the face of a tile's
// edge row is computed by two different warps).
__device__ __forceinline__ void recip4(double D0, double D1, double D2, double D3, double &i0,
                                       double &i1, double &i2, double &i3)
{
    const double p01 = __dmul_rn(D0, D1), p23 = __dmul_rn(D2, D3);
    const double r = 1.0 / __dmul_rn(p01, p23);
    const double r01 = __dmul_rn(r, p23), r23 = __dmul_rn(r, p01);
    i0 = __dmul_rn(r01, D1);
    i1 = __dmul_rn(r01, D0);
    i2 = __dmul_rn(r23, D3);
    i3 = __dmul_rn(r23, D2);
}

// FP32-bulk form: the face value minus the centre value from the six
// stencil differences A..G = u[-3..3] - u[0] (skipping the centre), which the
// caller takes in FP64 so that FP32 sees only the small differences and not
// the O(1) values.  Same indicators, candidates and weights as above; the
// weights use fast reciprocals.
__device__ __forceinline__ float weno7_corr(float A, float B, float Cc, float E, float F, float G)
{
    const float eps = 1e-6f;
    float s0 = E * (11003.f * E - 17246.f * F + 4642.f * G) + F * (7043.f * F - 3882.f * G) +
               547.f * G * G;
    float s1 = Cc * (547.f * Cc + 1922.f * E - 494.f * F) + E * (2843.f * E - 1642.f * F) +
               267.f * F * F;
    float s2 = B * (267.f * B - 1642.f * Cc - 494.f * E) + Cc * (2843.f * Cc + 1922.f * E) +
               547.f * E * E;
    float s3 = A * (547.f * A - 3882.f * B + 4642.f * Cc) + B * (7043.f * B - 17246.f * Cc) +
               11003.f * Cc * Cc;
    float q0 = 13.f * E - 5.f * F + G;
    float q1 = -Cc + 7.f * E - F;
    float q2 = B - 5.f * Cc + 3.f * E;
    float q3 = -3.f * A + 13.f * B - 23.f * Cc;
    float w0 = __fdividef(4.f, (eps + s0) * (eps + s0));
    float w1 = __fdividef(18.f, (eps + s1) * (eps + s1));
    float w2 = __fdividef(12.f, (eps + s2) * (eps + s2));
    float w3 = __fdividef(1.f, (eps + s3) * (eps + s3));
    float num = w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3;
    return __fdividef(num, 12.f * (w0 + w1 + w2 + w3));
}

}  // namespace cosenu
