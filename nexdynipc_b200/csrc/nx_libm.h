// nx_libm.h — portable FP64 elementary functions shared by the CPU oracle and
// the device code, so that both sides round every operation identically.
//
// Written from the mathematics: Cody & Waite style additive argument
// reduction (pi/2 and ln 2 split into short-mantissa parts so that k*part
// is exact) followed by truncated Taylor series whose coefficients are the
// exact rationals 1/n!, 1/(2k+1), 2/(2k+1) rounded once to double.  Series
// lengths leave truncation errors below 1e-19 relative on the reduced
// ranges, so the results stay within a few ulp of the correctly rounded
// value (tests/test_libm.py measures this against the C library).
// Only +, -, *, /, sqrt, frexp/ldexp and comparisons are used; compile
// without FMA contraction (nvcc --fmad=false, g++ -ffp-contract=off).
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define NXM_HD __host__ __device__ __forceinline__
#else
#define NXM_HD inline
#endif

namespace nxm {

// pi/2 = PIO2_1 + PIO2_2 + PIO2_3 (32 + 32 + 53 significant bits)
constexpr double PIO2_1 = 1.5707963267341256;
constexpr double PIO2_2 = 6.077100506303966e-11;
constexpr double PIO2_3 = 2.0222662487959506e-21;
constexpr double TWO_OVER_PI = 0.6366197723675814;
constexpr double PIO2_HI = 1.5707963267948966, PIO2_LO = 6.123233995736766e-17;
constexpr double PIO6_HI = 0.5235987755982989, PIO6_LO = -5.360408832255455e-17;
constexpr double SQRT3 = 1.7320508075688772;
constexpr double TAN_PI_12 = 0.2679491924311227;
constexpr double SQRT_HALF = 0.7071067811865476;
// ln 2 = LN2_HI + LN2_LO (32 + 53 bits)
constexpr double LN2_HI = 0.6931471803691238, LN2_LO = 1.9082149292705877e-10;
constexpr double INV_LN2 = 1.4426950408889634;

NXM_HD double round_half_away(double v) { return v >= 0.0 ? floor(v + 0.5) : -floor(-v + 0.5); }

// sin(r), cos(r) for |r| <= pi/4
NXM_HD double sin_kernel(double r) {
    const double z = r * r;
    return r + r * z * (-0.16666666666666666 + z * (0.008333333333333333 + z * (-0.0001984126984126984 + z * (2.7557319223985893e-06 + z * (-2.505210838544172e-08 + z * (1.6059043836821613e-10 + z * (-7.647163731819816e-13 + z * (2.8114572543455206e-15 + z * (-8.22063524662433e-18 + z * (1.9572941063391263e-20))))))))));
}
NXM_HD double cos_kernel(double r) {
    const double z = r * r;
    return 1.0 + z * (-0.5 + z * (0.041666666666666664 + z * (-0.001388888888888889 + z * (2.48015873015873e-05 + z * (-2.755731922398589e-07 + z * (2.08767569878681e-09 + z * (-1.1470745597729725e-11 + z * (4.779477332387385e-14 + z * (-1.5619206968586225e-16 + z * (4.110317623312165e-19 + z * (-8.896791392450574e-22)))))))))));
}

NXM_HD void sincos(double x, double* s, double* c) {
    if (!(fabs(x) <= 1.7976931348623157e308)) {   // inf or nan
        *s = x - x; *c = x - x;
        return;
    }
    // k * PIO2_1 and k * PIO2_2 are exact for |k| < 2^21 (|x| < 3e6); larger
    // arguments are reduced inexactly (identically on host and device)
    double r = x;
    int q = 0;
    if (fabs(x) > 0.7853981633974483) {
        const double k = round_half_away(x * TWO_OVER_PI);
        r = ((x - k * PIO2_1) - k * PIO2_2) - k * PIO2_3;
        q = ((long long)k) & 3;
    }
    const double sr = sin_kernel(r), cr = cos_kernel(r);
    switch (q) {
        case 0: *s = sr; *c = cr; break;
        case 1: *s = cr; *c = -sr; break;
        case 2: *s = -sr; *c = -cr; break;
        default: *s = -cr; *c = sr; break;
    }
}
NXM_HD double sin(double x) { double s, c; sincos(x, &s, &c); return s; }
NXM_HD double cos(double x) { double s, c; sincos(x, &s, &c); return c; }

// atan(u) for |u| <= tan(pi/12)
NXM_HD double atan_kernel(double u) {
    const double z = u * u;
    return u + u * z * (-0.3333333333333333 + z * (0.2 + z * (-0.14285714285714285 + z * (0.1111111111111111 + z * (-0.09090909090909091 + z * (0.07692307692307693 + z * (-0.06666666666666667 + z * (0.058823529411764705 + z * (-0.05263157894736842 + z * (0.047619047619047616 + z * (-0.043478260869565216 + z * (0.04 + z * (-0.037037037037037035 + z * (0.034482758620689655 + z * (-0.03225806451612903)))))))))))))));
}
// atan(t) for 0 <= t <= 1, returned as hi + lo
NXM_HD double atan01(double t) {
    if (t <= TAN_PI_12) return atan_kernel(t);
    // atan(t) = pi/6 + atan((sqrt3 t - 1) / (t + sqrt3))
    const double u = (t * SQRT3 - 1.0) / (t + SQRT3);
    return PIO6_HI + (PIO6_LO + atan_kernel(u));
}
NXM_HD double atan2(double y, double x) {
    if (x != x || y != y) return x + y;
    const double ax = fabs(x), ay = fabs(y);
    double a;
    if (ay == 0.0 && ax == 0.0) a = 0.0;
    else if (ay <= ax) a = atan01(ay / ax);
    else a = PIO2_HI + (PIO2_LO - atan01(ax / ay));
    if (x < 0.0) a = (PIO2_HI + PIO2_HI) + ((PIO2_LO + PIO2_LO) - a);
    return y < 0.0 ? -a : a;
}

NXM_HD double log(double x) {
    if (!(x > 0.0)) return x == 0.0 ? -INFINITY : (x - x) / (x - x);
    if (x == INFINITY) return x;
    int e;
    double m = frexp(x, &e);          // x = m 2^e, m in [0.5, 1)
    if (m < SQRT_HALF) { m = m + m; e -= 1; }
    const double f = (m - 1.0) / (m + 1.0);
    const double z = f * f;
    const double lm = (f + f) + f * z * (0.6666666666666666 + z * (0.4 + z * (0.2857142857142857 + z * (0.2222222222222222 + z * (0.18181818181818182 + z * (0.15384615384615385 + z * (0.13333333333333333 + z * (0.11764705882352941 + z * (0.10526315789473684 + z * (0.09523809523809523 + z * (0.08695652173913043 + z * (0.08))))))))))));
    const double k = (double)e;
    return k * LN2_HI + (k * LN2_LO + lm);
}

NXM_HD double exp(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return INFINITY;
    if (x < -745.1332191019412) return 0.0;
    const double k = round_half_away(x * INV_LN2);
    const double r = (x - k * LN2_HI) - k * LN2_LO;
    const double p = 1.0 + (r + r * r * (0.5 + r * (0.16666666666666666 + r * (0.041666666666666664 + r * (0.008333333333333333 + r * (0.001388888888888889 + r * (0.0001984126984126984 + r * (2.48015873015873e-05 + r * (2.7557319223985893e-06 + r * (2.755731922398589e-07 + r * (2.505210838544172e-08 + r * (2.08767569878681e-09 + r * (1.6059043836821613e-10 + r * (1.1470745597729725e-11 + r * (7.647163731819816e-13)))))))))))))));
    return ldexp(p, (int)k);
}

// exp(y) - 1 for |y| <= 1
NXM_HD double expm1_small(double y) {
    return y + y * y * (0.5 + y * (0.16666666666666666 + y * (0.041666666666666664 + y * (0.008333333333333333 + y * (0.001388888888888889 + y * (0.0001984126984126984 + y * (2.48015873015873e-05 + y * (2.7557319223985893e-06 + y * (2.755731922398589e-07 + y * (2.505210838544172e-08 + y * (2.08767569878681e-09 + y * (1.6059043836821613e-10 + y * (1.1470745597729725e-11 + y * (7.647163731819816e-13 + y * (4.779477332387385e-14 + y * (2.8114572543455206e-15 + y * (1.5619206968586225e-16 + y * (8.22063524662433e-18 + y * (4.110317623312165e-19 + y * (1.9572941063391263e-20))))))))))))))))))));
}

NXM_HD double tanh(double s) {
    const double a = fabs(s);
    double t;
    if (a > 20.0) t = 1.0;
    else if (a < 0.5) { const double em = expm1_small(a + a); t = em / (em + 2.0); }
    else { const double e = exp(a + a); t = 1.0 - 2.0 / (e + 1.0); }
    return s < 0.0 ? -t : t;
}

NXM_HD double cosh(double s) {
    const double e = exp(fabs(s));
    return 0.5 * (e + 1.0 / e);
}

}  // namespace nxm
