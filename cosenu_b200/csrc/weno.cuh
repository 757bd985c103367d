// WENO7 face reconstruction shared by the stage kernels.
#pragma once

#include "common.cuh"

namespace cosenu {

// WENO7 face value from the 7-point stencil a..g = u[-3..3] about the cell
// whose right face (j+1/2) is reconstructed with left-biased weights
// (rflux of src/rhs_fv.hpp:37-71).  Smoothness indicators and candidate
// polynomials of the four 4-point sub-stencils; nonlinear weights
// gamma_r / (eps + beta_r)^2 with gamma = (4, 18, 12, 1)/35 and eps = 1e-6.
// FP64: the four weights are brought to a common denominator so that the
// face needs one division.
__device__ __forceinline__ double weno7_face(double a, double b, double c, double d, double e,
                                             double f, double g)
{
    const double eps = 1e-6;
    double s0 = d * (2107. * d - 9402. * e + 7042. * f - 1854. * g) +
                e * (11003. * e - 17246. * f + 4642. * g) + f * (7043. * f - 3882. * g) +
                547. * g * g;
    double s1 = c * (547. * c - 2522. * d + 1922. * e - 494. * f) +
                d * (3443. * d - 5966. * e + 1602. * f) + e * (2843. * e - 1642. * f) +
                267. * f * f;
    double s2 = b * (267. * b - 1642. * c + 1602. * d - 494. * e) +
                c * (2843. * c - 5966. * d + 1922. * e) + d * (3443. * d - 2522. * e) +
                547. * e * e;
    double s3 = a * (547. * a - 3882. * b + 4642. * c - 1854. * d) +
                b * (7043. * b - 17246. * c + 7042. * d) + c * (11003. * c - 9402. * d) +
                2107. * d * d;
    // 12 x candidate values
    double q0 = 3. * d + 13. * e - 5. * f + g;
    double q1 = -c + 7. * d + 7. * e - f;
    double q2 = b - 5. * c + 13. * d + 3. * e;
    double q3 = -3. * a + 13. * b - 23. * c + 25. * d;
    double d0 = (eps + s0) * (eps + s0);
    double d1 = (eps + s1) * (eps + s1);
    double d2 = (eps + s2) * (eps + s2);
    double d3 = (eps + s3) * (eps + s3);
    double d01 = d0 * d1, d23 = d2 * d3;
    double w0 = 4. * d1 * d23;
    double w1 = 18. * d0 * d23;
    double w2 = 12. * d01 * d3;
    double w3 = d01 * d2;
    double num = w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3;
    double den = 12. * (w0 + w1 + w2 + w3);
    return num / den;
}

// FP32 variant: the indicators are evaluated on differences from the centre
// value (they are invariant under a constant shift, which removes the
// cancellation that FP32 would otherwise suffer on O(1) data), and the weights
// use fast reciprocals.
__device__ __forceinline__ float weno7_face(float a, float b, float c, float d, float e, float f,
                                            float g)
{
    const float eps = 1e-6f;
    float A = a - d, B = b - d, Cc = c - d, E = e - d, F = f - d, G = g - d;
    float s0 = E * (11003.f * E - 17246.f * F + 4642.f * G) + F * (7043.f * F - 3882.f * G) +
               547.f * G * G;
    float s1 = Cc * (547.f * Cc + 1922.f * E - 494.f * F) + E * (2843.f * E - 1642.f * F) +
               267.f * F * F;
    float s2 = B * (267.f * B - 1642.f * Cc - 494.f * E) + Cc * (2843.f * Cc + 1922.f * E) +
               547.f * E * E;
    float s3 = A * (547.f * A - 3882.f * B + 4642.f * Cc) + B * (7043.f * B - 17246.f * Cc) +
               11003.f * Cc * Cc;
    float q0 = 3.f * d + 13.f * e - 5.f * f + g;
    float q1 = -c + 7.f * d + 7.f * e - f;
    float q2 = b - 5.f * c + 13.f * d + 3.f * e;
    float q3 = -3.f * a + 13.f * b - 23.f * c + 25.f * d;
    float w0 = __fdividef(4.f, (eps + s0) * (eps + s0));
    float w1 = __fdividef(18.f, (eps + s1) * (eps + s1));
    float w2 = __fdividef(12.f, (eps + s2) * (eps + s2));
    float w3 = __fdividef(1.f, (eps + s3) * (eps + s3));
    float num = w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3;
    return __fdividef(num, 12.f * (w0 + w1 + w2 + w3));
}

}  // namespace cosenu
