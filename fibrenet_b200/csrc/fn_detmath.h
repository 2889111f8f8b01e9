/*
 * fn_detmath.h -- arc cosine built only from IEEE-754 +, -, *, / and sqrt,
 * so the device and a host checker produce bit-identical results (provided
 * neither contracts a*b+c into an FMA: nvcc -fmad=false, gcc
 * -ffp-contract=off).  Library acos implementations differ between CUDA and
 * glibc in the last bit, which would make long trajectories diverge bitwise.
 *
 * Method (the classical half-angle reduction for arcsine):
 *   asin(s) = s + s^3 R(s^2),           0 <= s <= 1/2
 *   acos(x) = pi/2 - asin(x),           |x| <= 1/2
 *   acos(x) = 2 asin(sqrt((1-x)/2)),     x  >  1/2
 *   acos(x) = pi - 2 asin(sqrt((1+x)/2)), x < -1/2
 * R(z) = (asin(sqrt z) - sqrt z) / z^1.5 on [0, 1/4] is replaced by its
 * degree-13 interpolant at the Chebyshev points of the first kind (60-digit
 * arithmetic with mpmath, written in monomial form and rounded to doubles;
 * tests/detmath_fit.py regenerates the coefficients); the interpolation
 * error is below 3e-19 relative to asin, so the result is within a few ulp
 * of acos.
 */
#ifndef FIBRENET_DETMATH_H
#define FIBRENET_DETMATH_H

#if defined(__CUDACC__)
#define FN_HD __host__ __device__ __forceinline__
#else
#define FN_HD static inline
#endif

#include <math.h>

FN_HD double fn_asin_poly(double s) {
    const double c[14] = {
        0.16666666666666666,
        0.07500000000000118,
        0.044642857142551895,
        0.03038194447553234,
        0.02237215744350722,
        0.017352816540325496,
        0.01396378001220357,
        0.011566459612121669,
        0.009621842970100282,
        0.009319560794767446,
        0.0030448799094556773,
        0.019554513336123378,
        -0.01924167174674304,
        0.02961201126495512};
    double z = s * s;
    double r = c[13];
    for (int k = 12; k >= 0; --k) r = r * z + c[k];
    return s + (s * z) * r;
}

FN_HD double fn_acos(double x) {
    const double pi = 3.141592653589793;
    const double half_pi = 1.5707963267948966;
    if (x != x) return x;
    if (x > 0.5) {
        double s = sqrt((1.0 - x) * 0.5);
        return 2.0 * fn_asin_poly(s);
    }
    if (x < -0.5) {
        double s = sqrt((1.0 + x) * 0.5);
        return pi - 2.0 * fn_asin_poly(s);
    }
    return half_pi - fn_asin_poly(x);
}

#endif
