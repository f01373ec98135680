// ORACLE — test infrastructure only (see abm3d.hpp).
//
// Deterministic log, sin and cos for the division draws.  The draw policy
// (Philox counters feeding Box-Muller normals and uniform angles) is shared with
// the CUDA path, and two daughters of one mother are placed exactly 2R apart
// end to end, where the JKR force jumps at zero overlap: a one-ulp difference in
// a daughter length decides whether the siblings touch.  So both sides evaluate
// these functions with the same sequence of correctly rounded operations
// (this file is compiled with -ffp-contract=off):
//   log x   frexp range reduction to m in [sqrt(1/2), sqrt(2)), then
//           log m = 2 atanh((m - 1)/(m + 1)) by its power series (to f^29);
//   sin/cos Cody-Waite reduction by pi/2 with a two-part constant, then the
//           Taylor series of sin and cos on [-pi/4, pi/4] (to r^23 / r^22).
// The two-part constants ln 2 = LN2_HI + LN2_LO and pi/2 = PIO2_HI + PIO2_LO are the
// published split values of fdlibm (Sun Microsystems, 1993: e_log.c and e_rem_pio2.c).
#pragma once
#include <cmath>

namespace oracle {

const double DET_LN2_HI = 6.93147180369123816490e-01;
const double DET_LN2_LO = 1.90821492927058770002e-10;
const double DET_SQRT_HALF = 0.70710678118654752440;
const double DET_TWO_OVER_PI = 0.63661977236758134308;
const double DET_PIO2_HI = 1.57079632673412561417e+00;
const double DET_PIO2_LO = 6.07710050650619224932e-11;

inline double det_log(double x)
{
    int e;
    double m = std::frexp(x, &e);
    if (m < DET_SQRT_HALF) { m = m * 2.0; e = e - 1; }
    double f = (m - 1.0) / (m + 1.0);
    double f2 = f * f;
    double p = 1.0 / 29.0;
    for (int k = 27; k >= 1; k -= 2) p = p * f2 + 1.0 / (double)k;
    double ed = (double)e;
    return ed * DET_LN2_HI + (2.0 * f * p + ed * DET_LN2_LO);
}

inline void det_sincos(double x, double& s, double& c)
{
    double k = std::rint(x * DET_TWO_OVER_PI);
    double r = (x - k * DET_PIO2_HI) - k * DET_PIO2_LO;
    double r2 = r * r;
    // sin r = r (1 - r^2/3! + r^4/5! - ...), cos r = 1 - r^2/2! + r^4/4! - ...
    double ps = 1.0, pc = 1.0;
    for (int n = 22; n >= 2; n -= 2)
    {
        ps = 1.0 - ps * r2 / (double)((n + 1) * n);
        pc = 1.0 - pc * r2 / (double)(n * (n - 1));
    }
    double sr = r * ps, cr = pc;
    int q = (int)((long long)k & 3);
    if (q == 0) { s = sr; c = cr; }
    else if (q == 1) { s = cr; c = -sr; }
    else if (q == 2) { s = -sr; c = -cr; }
    else { s = -cr; c = sr; }
}

}   // namespace oracle
