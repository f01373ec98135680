// Device-side building blocks of the B200 mechanics step: state records,
// exact-rounding segment distance, surface integrals, the per-cell velocity
// solve and the Philox counter RNG.  Every function names the reference
// file:line (kmnam/biofilm-ABMs, ABM-3d/ABM-3d-cpp/include) whose arithmetic
// it reproduces.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace abm {

// ---------------------------------------------------------------------------
// State records.  Cell geometry is gathered at random by the pair kernels, so
// it is one 64-byte record per cell (two 32-byte sectors, read as four 16-byte
// loads); everything else is streamed once per cell per kernel.
// ---------------------------------------------------------------------------
struct __align__(64) Geom {     // position, half-length, orientation, gamma
    double rx, ry, rz, h;
    double nx, ny, nz, gamma;
};
struct __align__(16) Vel {      // stored velocities of the last accepted step (dr, dn)
    double v[6];
};
struct __align__(64) Phys {     // l, growth, eta0, eta1, sigma0, t0, id, group
    double l, growth, eta0, eta1, sigma0, t0, id, group;
};
struct __align__(16) Gen6 {     // generalised force / dE/dq
    double f[6];
};

__device__ __forceinline__ Geom load_geom(const Geom* __restrict__ g, int i)
{
    const double2* p = reinterpret_cast<const double2*>(g + i);
    double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    Geom o;
    o.rx = a.x; o.ry = a.y; o.rz = b.x; o.h = b.y;
    o.nx = c.x; o.ny = c.y; o.nz = d.x; o.gamma = d.y;
    return o;
}

// Rigorous lower bound test on the distance of two segments: false only when the
// gap between their projections on the single-precision closest-point direction a,
//     a . (c_b - c_a) - h_a |a . n_a| - h_b |a . n_b|   (FP64),
// exceeds limit + 1e-9.  For any unit a that gap bounds the distance from below,
// and the reference's distance (CGAL's minimiser, or the near-parallel branch's
// feasible pair of points) is never below the true minimum, so a pair that fails
// the test is farther than `limit` in the reference too.
__device__ __forceinline__ bool may_touch(const Geom& a, const Geom& b, double limit)
{
    const double wx = b.rx - a.rx, wy = b.ry - a.ry, wz = b.rz - a.rz;
    // single-precision closest points (clamped, one refinement): only a direction
    const float fwx = (float)wx, fwy = (float)wy, fwz = (float)wz;
    const float ax = (float)a.nx, ay = (float)a.ny, az = (float)a.nz;
    const float bx = (float)b.nx, by = (float)b.ny, bz = (float)b.nz;
    const float ha = (float)a.h, hb = (float)b.h;
    const float B = ax * bx + ay * by + az * bz;
    const float D = ax * fwx + ay * fwy + az * fwz, E = bx * fwx + by * fwy + bz * fwz;
    const float den = 1.f - B * B;
    float s = den > 1e-6f ? (D - B * E) / den : 0.f;
    s = fminf(fmaxf(s, -ha), ha);
    float t = fminf(fmaxf(B * s - E, -hb), hb);
    s = fminf(fmaxf(B * t + D, -ha), ha);
    const double dx = wx + (double)t * b.nx - (double)s * a.nx;
    const double dy = wy + (double)t * b.ny - (double)s * a.ny;
    const double dz = wz + (double)t * b.nz - (double)s * a.nz;
    const double dn = sqrt(dx * dx + dy * dy + dz * dz);
    if (!(dn > 1e-6)) return true;
    const double ux = dx / dn, uy = dy / dn, uz = dz / dn;
    const double gap = (ux * wx + uy * wy + uz * wz) - a.h * fabs(ux * a.nx + uy * a.ny + uz * a.nz)
                       - b.h * fabs(ux * b.nx + uy * b.ny + uz * b.nz);
    return !(gap > limit + 1e-9);
}

// ---------------------------------------------------------------------------
// Exact-rounding vector arithmetic.  The neighbor decision |d| < threshold
// must come out identically on the GPU and in the CPU restatement, so the
// segment distance uses only correctly rounded +, -, *, /, sqrt with no
// fused multiply-add (the __d*_rn intrinsics are never contracted), summing
// dot products as ((x + y) + z).
// ---------------------------------------------------------------------------
struct X3 { double x, y, z; };
__device__ __forceinline__ X3 x3(double x, double y, double z) { X3 v; v.x = x; v.y = y; v.z = z; return v; }
__device__ __forceinline__ X3 xadd(X3 a, X3 b) { return x3(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y), __dadd_rn(a.z, b.z)); }
__device__ __forceinline__ X3 xsub(X3 a, X3 b) { return x3(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)); }
__device__ __forceinline__ X3 xscale(double s, X3 a) { return x3(__dmul_rn(s, a.x), __dmul_rn(s, a.y), __dmul_rn(s, a.z)); }
__device__ __forceinline__ double xdot(X3 a, X3 b)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z));
}
__device__ __forceinline__ double xnorm(X3 a) { return __dsqrt_rn(xdot(a, a)); }

// distances.hpp:92-105 (nearestCellBodyCoordToPoint)
__device__ __forceinline__ double nearest_body_coord(X3 r, X3 n, double h, X3 q)
{
    double s = xdot(xsub(q, r), n);
    if (fabs(s) <= h) return s;
    else if (s > h) return h;
    return -h;
}

__device__ __forceinline__ double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

// Closest-point parameters of two segments p1 + x (q1 - p1), p2 + y (q2 - p2),
// standing in for CGAL's Segment_3/Segment_3 squared_distance result
// (distances.hpp:341).  Method: Ericson, Real-Time Collision Detection (2005),
// sec. 5.1.9.
__device__ __forceinline__ void closest_params(X3 p1, X3 q1, X3 p2, X3 q2, double& x, double& y)
{
    X3 d1 = xsub(q1, p1), d2 = xsub(q2, p2), r = xsub(p1, p2);
    double a = xdot(d1, d1), e = xdot(d2, d2), f = xdot(d2, r);
    if (a <= 0.0 && e <= 0.0) { x = 0.0; y = 0.0; return; }
    if (a <= 0.0) { x = 0.0; y = clamp01(__ddiv_rn(f, e)); return; }
    double c = xdot(d1, r);
    if (e <= 0.0) { y = 0.0; x = clamp01(__ddiv_rn(-c, a)); return; }
    double b = xdot(d1, d2);
    double denom = __dsub_rn(__dmul_rn(a, e), __dmul_rn(b, b));
    double s = (denom != 0.0)
        ? clamp01(__ddiv_rn(__dsub_rn(__dmul_rn(b, f), __dmul_rn(c, e)), denom)) : 0.0;
    double t = __ddiv_rn(__dadd_rn(__dmul_rn(b, s), f), e);
    if (t < 0.0) { t = 0.0; s = clamp01(__ddiv_rn(-c, a)); }
    else if (t > 1.0) { t = 1.0; s = clamp01(__ddiv_rn(__dsub_rn(b, c), a)); }
    x = s; y = t;
}

struct Dist { double dx, dy, dz, s, t; };

// distances.hpp:227-337: the near-parallel branch (|n1 . n2| >= 0.9999), kept out
// of line so the common skew path keeps its registers
static __device__ __noinline__ Dist dist_near_parallel(X3 r1, X3 n1, double h1, X3 r2, X3 n2, double h2)
{
    X3 p1 = xsub(r1, xscale(h1, n1)), q1 = xadd(r1, xscale(h1, n1));
    X3 p2 = xsub(r2, xscale(h2, n2)), q2 = xadd(r2, xscale(h2, n2));
    X3 d; double s, t;
        double s_p1 = nearest_body_coord(r2, n2, h2, p1);
        double s_q1 = nearest_body_coord(r2, n2, h2, q1);
        X3 d_p1 = xsub(xadd(r2, xscale(s_p1, n2)), p1);
        X3 d_q1 = xsub(xadd(r2, xscale(s_q1, n2)), q1);
        double dist_p1 = xnorm(d_p1), dist_q1 = xnorm(d_q1);
        if (s_p1 == s_q1)
        {
            if (dist_p1 < dist_q1) { s = -h1; t = s_p1; d = d_p1; }
            else { s = h1; t = s_q1; d = d_q1; }
        }
        else
        {
            double s_p2 = nearest_body_coord(r1, n1, h1, p2);
            double s_q2 = nearest_body_coord(r1, n1, h1, q2);
            X3 d_p2 = xsub(xadd(r1, xscale(s_p2, n1)), p2);
            X3 d_q2 = xsub(xadd(r1, xscale(s_q2, n1)), q2);
            double dist_p2 = xnorm(d_p2), dist_q2 = xnorm(d_q2);
            // the two smallest of four distances; ties keep index order, as the
            // reference's std::sort of a 4-element range does (insertion sort):
            // element a lands at position #{b : d_b < d_a} + #{b < a : d_b == d_a}
            const double dv0 = dist_p1, dv1 = dist_q1, dv2 = dist_p2, dv3 = dist_q2;
            const int rk0 = (dv1 < dv0) + (dv2 < dv0) + (dv3 < dv0);
            const int rk1 = (dv0 <= dv1) + (dv2 < dv1) + (dv3 < dv1);
            const int rk2 = (dv0 <= dv2) + (dv1 <= dv2) + (dv3 < dv2);
            bool m0 = rk0 < 2, m1 = rk1 < 2;
            bool m2 = rk2 < 2;
            if (m0 && m1)
            {
                s = 0.0;
                t = nearest_body_coord(r2, n2, h2, r1);
                d = xsub(xadd(r2, xscale(t, n2)), r1);
            }
            else if (!m0 && !m1)
            {
                t = 0.0;
                s = nearest_body_coord(r1, n1, h1, r2);
                d = xsub(xsub(r2, r1), xscale(s, n1));
            }
            else
            {
                double end1 = m0 ? -h1 : h1;
                double end2 = m2 ? s_p2 : s_q2;
                s = __ddiv_rn(__dadd_rn(end1, end2), 2.0);
                t = nearest_body_coord(r2, n2, h2, xadd(r1, xscale(s, n1)));
                d = xsub(xsub(xadd(r2, xscale(t, n2)), r1), xscale(s, n1));
            }
        }
    
    Dist o;
    o.dx = d.x; o.dy = d.y; o.dz = d.z; o.s = s; o.t = t;
    return o;
}

// distances.hpp:206-357 (distBetweenCells): d runs from cell 1 to cell 2.
__device__ __forceinline__ Dist dist_between_cells(X3 r1, X3 n1, double h1, X3 r2, X3 n2, double h2)
{
    double cos_theta = xdot(n1, n2);
    if (cos_theta >= 0.9999 || cos_theta <= -0.9999) return dist_near_parallel(r1, n1, h1, r2, n2, h2);
    // skew: CGAL's segment closest points (distances.hpp:338-345)
    X3 p1 = xsub(r1, xscale(h1, n1)), q1 = xadd(r1, xscale(h1, n1));
    X3 p2 = xsub(r2, xscale(h2, n2)), q2 = xadd(r2, xscale(h2, n2));
    double x, y;
    closest_params(p1, q1, p2, q2, x, y);
    double s = __dsub_rn(__dmul_rn(__dmul_rn(x, 2.0), h1), h1);
    double t = __dsub_rn(__dmul_rn(__dmul_rn(y, 2.0), h2), h2);
    X3 d = xsub(xsub(xadd(r2, xscale(t, n2)), r1), xscale(s, n1));
    Dist o;
    o.dx = d.x; o.dy = d.y; o.dz = d.z; o.s = s; o.t = t;
    return o;
}

__device__ __forceinline__ Dist dist_geom(const Geom& a, const Geom& b)
{
    return dist_between_cells(x3(a.rx, a.ry, a.rz), x3(a.nx, a.ny, a.nz), a.h,
                              x3(b.rx, b.ry, b.rz), x3(b.nx, b.ny, b.nz), b.h);
}

// Mixed-precision variant: the generic (skew) branch in FP32, the
// near-parallel branch (|cos| >= 0.9999, ill-conditioned s, t) in FP64.
__device__ __forceinline__ Dist dist_geom_mixed(const Geom& a, const Geom& b)
{
    float n1x = (float)a.nx, n1y = (float)a.ny, n1z = (float)a.nz;
    float n2x = (float)b.nx, n2y = (float)b.ny, n2z = (float)b.nz;
    double cos_theta = xdot(x3(a.nx, a.ny, a.nz), x3(b.nx, b.ny, b.nz));
    // FP64 for the near-parallel branch (|cos| >= 0.9999) and for the skew pairs just
    // short of it: the FP32 solve divides by a e - b^2 ~ (1 - cos^2) a e, which loses
    // 1/(1 - cos^2) of its digits, and the distance error, second order in (s, t),
    // stays below FP32 rounding of the overlap only for |cos| < 0.99
    if (cos_theta >= 0.99 || cos_theta <= -0.99) return dist_geom(a, b);
    // relative coordinates keep FP32 well conditioned far from the origin
    float rx = (float)(b.rx - a.rx), ry = (float)(b.ry - a.ry), rz = (float)(b.rz - a.rz);
    float h1 = (float)a.h, h2 = (float)b.h;
    // segment 1: -h1 n1 .. +h1 n1 (origin at r1); segment 2: r - h2 n2 .. r + h2 n2
    float d1x = 2.f * h1 * n1x, d1y = 2.f * h1 * n1y, d1z = 2.f * h1 * n1z;
    float d2x = 2.f * h2 * n2x, d2y = 2.f * h2 * n2y, d2z = 2.f * h2 * n2z;
    float p2x = rx - h2 * n2x, p2y = ry - h2 * n2y, p2z = rz - h2 * n2z;
    float wx = -h1 * n1x - p2x, wy = -h1 * n1y - p2y, wz = -h1 * n1z - p2z;   // p1 - p2
    float aa = d1x * d1x + d1y * d1y + d1z * d1z;
    float e = d2x * d2x + d2y * d2y + d2z * d2z;
    float f = d2x * wx + d2y * wy + d2z * wz;
    float c = d1x * wx + d1y * wy + d1z * wz;
    float bb = d1x * d2x + d1y * d2y + d1z * d2z;
    float x, y;
    if (aa <= 0.f && e <= 0.f) { x = 0.f; y = 0.f; }
    else if (aa <= 0.f) { x = 0.f; y = fminf(fmaxf(f / e, 0.f), 1.f); }
    else if (e <= 0.f) { y = 0.f; x = fminf(fmaxf(-c / aa, 0.f), 1.f); }
    else
    {
        float denom = aa * e - bb * bb;
        float s = denom != 0.f ? fminf(fmaxf((bb * f - c * e) / denom, 0.f), 1.f) : 0.f;
        float t = (bb * s + f) / e;
        if (t < 0.f) { t = 0.f; s = fminf(fmaxf(-c / aa, 0.f), 1.f); }
        else if (t > 1.f) { t = 1.f; s = fminf(fmaxf((bb - c) / aa, 0.f), 1.f); }
        x = s; y = t;
    }
    // the closest-point parameters come from the FP32 solve; the distance vector is
    // assembled from them in FP64.  Its length is stationary in (s, t) at an interior
    // minimum, and a clamped parameter is exact, so the overlap 2R - |d| keeps close to
    // FP64 accuracy instead of losing the 2^-24 |d| that an FP32 |d| ~ 2R would cost it.
    const double s1 = (double)x * 2.0 * a.h - a.h, t2 = (double)y * 2.0 * b.h - b.h;
    Dist o;
    o.dx = ((b.rx - a.rx) + t2 * b.nx) - s1 * a.nx;
    o.dy = ((b.ry - a.ry) + t2 * b.ny) - s1 * a.ny;
    o.dz = ((b.rz - a.rz) + t2 * b.nz) - s1 * a.nz;
    o.s = s1; o.t = t2;
    return o;
}

// ---------------------------------------------------------------------------
// Deterministic log, sin, cos for the division draws.  Two daughters of one
// mother are placed exactly 2R apart end to end, where the JKR force jumps at
// zero overlap, so the draws must come out bit-identical in the CPU
// restatement: both evaluate the same sequence of correctly rounded operations.
//   log x   frexp reduction to m in [sqrt(1/2), sqrt(2)), log m = 2 atanh((m-1)/(m+1))
//           by its power series (to f^29);
//   sin/cos Cody-Waite reduction by pi/2 (two-part constant), Taylor series of sin
//           and cos on [-pi/4, pi/4] (to r^23 / r^22).
// The two-part constants ln 2 = LN2_HI + LN2_LO and pi/2 = PIO2_HI + PIO2_LO are the
// published split values of fdlibm (Sun Microsystems, 1993: e_log.c and e_rem_pio2.c).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double det_log(double x)
{
    const double LN2_HI = 6.93147180369123816490e-01, LN2_LO = 1.90821492927058770002e-10;
    int e;
    double m = frexp(x, &e);
    if (m < 0.70710678118654752440) { m = __dmul_rn(m, 2.0); e = e - 1; }
    double f = __ddiv_rn(__dsub_rn(m, 1.0), __dadd_rn(m, 1.0));
    double f2 = __dmul_rn(f, f);
    double p = __ddiv_rn(1.0, 29.0);
    for (int k = 27; k >= 1; k -= 2) p = __dadd_rn(__dmul_rn(p, f2), __ddiv_rn(1.0, (double)k));
    double ed = (double)e;
    return __dadd_rn(__dmul_rn(ed, LN2_HI), __dadd_rn(__dmul_rn(__dmul_rn(2.0, f), p), __dmul_rn(ed, LN2_LO)));
}

__device__ __forceinline__ void det_sincos(double x, double& s, double& c)
{
    const double TWO_OVER_PI = 0.63661977236758134308;
    const double PIO2_HI = 1.57079632673412561417e+00, PIO2_LO = 6.07710050650619224932e-11;
    double k = rint(__dmul_rn(x, TWO_OVER_PI));
    double r = __dsub_rn(__dsub_rn(x, __dmul_rn(k, PIO2_HI)), __dmul_rn(k, PIO2_LO));
    double r2 = __dmul_rn(r, r);
    double ps = 1.0, pc = 1.0;
    for (int n = 22; n >= 2; n -= 2)
    {
        ps = __dsub_rn(1.0, __ddiv_rn(__dmul_rn(ps, r2), (double)((n + 1) * n)));
        pc = __dsub_rn(1.0, __ddiv_rn(__dmul_rn(pc, r2), (double)(n * (n - 1))));
    }
    double sr = __dmul_rn(r, ps), cr = pc;
    int q = (int)((long long)k & 3);
    if (q == 0) { s = sr; c = cr; }
    else if (q == 1) { s = cr; c = -sr; }
    else if (q == 2) { s = -sr; c = -cr; }
    else { s = -cr; c = sr; }
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11), the counter-based draw policy shared
// with the CPU restatement.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r)
    {
        uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t y0 = hi1 ^ c[1] ^ k0, y2 = hi0 ^ c[3] ^ k1;
        c[0] = y0; c[1] = lo1; c[2] = y2; c[3] = lo0;
        k0 += W0; k1 += W1;
    }
}
__host__ __device__ __forceinline__ double philox_u01(uint32_t hi, uint32_t lo)
{
    uint64_t bits = (((uint64_t)hi << 32) | lo) >> 12;
    return ((double)bits + 0.5) * (1.0 / 4503599627370496.0);
}
const uint32_t RNG_PURPOSE_NOISE = 0x4E6F6973u;
const uint32_t RNG_PURPOSE_DIVIDE = 0x44697669u;
const uint32_t RNG_PURPOSE_SWITCH = 0x53776974u;

__host__ __device__ __forceinline__ double rng_uniform(uint64_t seed, uint32_t purpose, uint32_t a,
                                                       uint32_t b, uint32_t c, uint32_t d)
{
    uint32_t x[4] = {a, b, c, d};
    philox4x32_10(x, (uint32_t)seed, (uint32_t)(seed >> 32) ^ purpose);
    return philox_u01(x[0], x[1]);
}

// utils.hpp:648-655 (standardNormal, Box-Muller) on two policy uniforms, with the
// deterministic log / cos shared with the CPU restatement
__device__ __forceinline__ double std_normal(double u, double v)
{
    double s, c;
    det_sincos(__dmul_rn(6.283185307179586476925286766559005768, v), s, c);
    return __dmul_rn(__dsqrt_rn(__dmul_rn(-2.0, det_log(u))), c);
}

// ---------------------------------------------------------------------------
// Surface integrals (integrals.hpp) with the overlap powers taken from one
// square root per end: p^{k/2} = p^{floor(k/2)} (sqrt p)^{k mod 2}.
// ---------------------------------------------------------------------------
struct EndPow {               // end overlaps phi(-h) (p) and phi(+h) (q) and their roots
    double p, q, sp, sq;
};

// p^(e/2) for e = 1..7 (e = 2 (gamma + 1))
__device__ __forceinline__ double half_pow(double x, double sx, int e)
{
    double r = (e & 1) ? sx : 1.0;
    for (int k = 0; k < (e >> 1); ++k) r *= x;
    return r;
}
__device__ __forceinline__ double epw(const EndPow& w, int e, bool second)
{
    return second ? half_pow(w.q, w.sq, e) : half_pow(w.p, w.sp, e);
}

// integrals.hpp:116-140 (integral1) with gamma + 1 = e / 2; the division by
// nz (gamma + 1) is a multiplication by inz = 1 / nz and the constant 2 / e
__device__ __forceinline__ double integral1(const EndPow& w, double inz, double h, int e, double ss)
{
    const double ig1 = 2.0 / e;
    if (ss > h) return (epw(w, e, false) - epw(w, e, true)) * inz * ig1;
    else if (ss > -h) return epw(w, e, false) * inz * ig1;
    return 0.0;
}

// integrals.hpp:159-184 (integral2) with gamma + 1 = e / 2
__device__ __forceinline__ double integral2(const EndPow& w, double inz, double h, int e, double ss)
{
    double term1 = integral1(w, inz, h, e + 2, ss);
    double term2 = 0.0;
    if (ss > h) term2 = -h * (epw(w, e, false) + epw(w, e, true));
    else if (ss > -h) term2 = -h * epw(w, e, false);
    return (term1 + term2) * inz * (2.0 / e);
}

// The end overlaps that integral1/2 and areaIntegrals read (integrals.hpp:56-60,
// 431-441): both ends when ss > h, the lower end when -h < ss <= h.
__device__ __forceinline__ EndPow end_pows(double rz, double nz, double R, double h, double ss)
{
    EndPow w;
    w.p = 0.0; w.q = 0.0;
    if (ss > h) { w.p = R - rz - (-h) * nz; w.q = R - rz - h * nz; }
    else if (ss > -h) { w.p = R - rz - (-h) * nz; }
    w.sp = sqrt(w.p); w.sq = sqrt(w.q);
    return w;
}

struct MechParams {
    double R, Rcell, E0, Ecell;
    double sqrtR;
    double nz_threshold;
    double coulomb;          // cell_surface_coulomb_coeff
    int no_surface;
};

// The horizontal shortcut of the cell-surface forces (assume_2d): dE/dq component 2
// of repulsion and adhesion (mechanics.hpp:673-780 and 800-910)
__device__ __forceinline__ void surface_dEdq_flat(const MechParams& P, double rz, double l, double sigma0,
                                                  double& rep2, double& adh2)
{
    double ph = P.R - rz;
    if (ph > 0)
    {
        rep2 = -(2 * P.E0) * ph * l;
        adh2 = sigma0 * (P.sqrtR / 2) * l / sqrt(ph);
    }
}

// Cell-surface repulsion + adhesion dE/dq components 2 and 5
// (mechanics.hpp:673-780 and 800-910, include_constraint = false).
__device__ __forceinline__ void surface_dEdq(const MechParams& P, bool assume_2d, double rz, double nz,
                                             double l, double h, double sigma0, double ss,
                                             const EndPow& w, double& rep2, double& rep5,
                                             double& adh2, double& adh5)
{
    const double R = P.R, E0 = P.E0;
    rep2 = rep5 = adh2 = adh5 = 0.0;
    if (assume_2d)
    {
        surface_dEdq_flat(P, rz, l, sigma0, rep2, adh2);
        return;
    }
    const double pf0 = 2 * E0, pf1 = (8. / 3.) * E0 * P.sqrtR, pf2 = 2 * E0 * P.sqrtR;
    double nz2 = nz * nz;
    const double inz = 1.0 / nz;
    double int1 = integral1(w, inz, h, 4, ss);   // delta
    double int2 = integral1(w, inz, h, 3, ss);   // sqrt(delta)
    rep2 = -pf0 * ((1.0 - nz2) * int1 + P.sqrtR * nz2 * int2);
    double int3 = integral1(w, inz, h, 6, ss);   // delta^2
    double int4 = integral2(w, inz, h, 4, ss);   // s delta
    double int5 = integral1(w, inz, h, 5, ss);   // delta^1.5
    double int6 = integral2(w, inz, h, 3, ss);   // s sqrt(delta)
    double d5 = 0.0;
    d5 -= pf0 * nz * int3;
    d5 -= pf0 * (1 - nz2) * int4;
    d5 += pf1 * nz * int5;
    d5 -= pf2 * nz2 * int6;
    rep5 = d5;
    // adhesion
    const double a0 = P.sqrtR / 2, a1 = 2 * M_PI * R, a2 = 2 * P.sqrtR;
    double i1 = integral1(w, inz, h, 1, ss);     // delta^-1/2
    bool partial = fabs(ss) < h;
    double term2 = partial ? (a1 / 2) * nz : 0.0;
    adh2 = (a0 * (1 - nz2) * i1 + term2) * sigma0;
    double i2 = integral1(w, inz, h, 3, ss);     // delta^1/2
    double i3 = integral2(w, inz, h, 1, ss);     // s delta^-1/2
    double i4 = (ss > h) ? 2 * h : ((ss > -h) ? ss + h : 0.0);   // integral4
    double term4 = partial ? (a1 / 2) * (R - rz) : 0.0;
    double e5 = 0.0;
    e5 += a2 * nz * i2;
    e5 += a0 * (1 - nz2) * i3;
    e5 -= a1 * nz * i4;
    e5 += term4;
    adh5 = e5 * sigma0;
}

// integrals.hpp:400-463 (areaIntegrals)
__device__ __forceinline__ void area_integrals(const MechParams& P, double nz, double h, double ss,
                                               const EndPow& w, double& A1, double& A2, double& A3)
{
    const double R = P.R;
    double int4 = (ss > h) ? 2 * h : ((ss > -h) ? ss + h : 0.0);
    double int5 = (-h < ss && ss <= h) ? (ss * ss - h * h) / 2.0 : 0.0;
    double int6 = (ss > h) ? 2 * h * h * h / 3.0 : ((ss > -h) ? (ss * ss * ss + h * h * h) / 3.0 : 0.0);
    const double inz = 1.0 / nz;
    double int1a = integral1(w, inz, h, 3, ss);
    double int1b = integral1(w, inz, h, 5, ss);
    double int1c = integral1(w, inz, h, 7, ss);
    double onz = 1 - nz * nz;
    double piRnz2 = M_PI * R * nz * nz;
    A1 = P.sqrtR * onz * int1a + piRnz2 * int4;
    const double p3 = epw(w, 3, false), q3 = epw(w, 3, true);
    double term2 = -h * (p3 + q3);
    double int2a = (int1b + term2) * inz * (1.0 / 1.5);
    A2 = P.sqrtR * onz * int2a + piRnz2 * int5;
    term2 = -h * (epw(w, 5, false) + epw(w, 5, true));
    double int2b = (int1c + term2) * inz * (1.0 / 2.5);
    double int3 = (2 * int2b + h * h * (p3 - q3)) * inz * (1.0 / 1.5);
    A3 = P.sqrtR * onz * int3 + piRnz2 * int6;
}

// Does a cell touch the surface (mechanics.hpp:2080-2090)?
__device__ __forceinline__ bool surface_contact(const MechParams& P, bool assume_2d, const double y[6], double h)
{
    if (!assume_2d) return (y[2] - h * y[5] < P.R) || (y[2] + h * y[5] < P.R);
    return y[2] < P.R;
}

// The first two branches of getVelocities (mechanics.hpp:2011-2189): a cell clear of
// the surface, and a horizontal cell on it (assume_2d), with Coulomb truncation of the
// surface friction from the stored velocity dr of the previous accepted step.  Called
// only for those two kinds of cells, so a contacting cell here lies on the substrate.
__device__ __forceinline__ void velocity_free_or_flat(const MechParams& P, bool contacting, const double y[6],
                                                      double l, double eta0, double eta1_in,
                                                      const Vel* __restrict__ drp, const double f[6],
                                                      double v[6])
{
    const double R = P.R, E0 = P.E0, coul = P.coulomb;
    const double rz = y[2], nx = y[3], ny = y[4], nz = y[5];
    if (P.no_surface || !contacting)
    {
        double K = eta0 * l, L = K * l * l / 12;
        double mult = -((nx * f[3] + ny * f[4]) + nz * f[5]);
        v[0] = f[0] / K; v[1] = f[1] / K; v[2] = f[2] / K;
        v[3] = (f[3] + mult * nx) / L; v[4] = (f[4] + mult * ny) / L; v[5] = (f[5] + mult * nz) / L;
    }
    else
    {
        double K, L;
        double a = sqrt(R * (R - rz));
        if (coul == 0)
        {
            double eta_c = eta0 + eta1_in * a / R;
            K = eta_c * l; L = K * l * l / 12;
        }
        else
        {
            double K_vis = eta0 * l, L_vis = K_vis * l * l / 12;
            double K_fric = eta1_in * l * a / R;
            const double2 d01 = __ldg(reinterpret_cast<const double2*>(drp->v));
            double drxy = sqrt(d01.x * d01.x + d01.y * d01.y);
            double max_norm = coul * (2 * E0 * (R - rz) * l);
            if (K_fric * drxy > max_norm)
            {
                double eta1_tr = max_norm * R / (drxy * l * a);
                K_fric = eta1_tr * l * a / R;
            }
            K = K_vis + K_fric; L = L_vis + K_fric * l * l / 12;
        }
        double mult = -(nx * f[3] + ny * f[4]);
        v[0] = f[0] / K; v[1] = f[1] / K;
        v[3] = (f[3] + mult * nx) / L; v[4] = (f[4] + mult * ny) / L;
        v[2] = f[2] / (eta0 * l);
        v[5] = 12 * f[5] / (eta0 * l * l * l);
    }
}

// Velocity of one cell from its generalised force (mechanics.hpp:2011-2347,
// the three branches: no surface contact, horizontal contact, full 3-D contact).
// dr, dn: stored velocities of the previous accepted step (Coulomb truncation).
__device__ __forceinline__ void velocity_solve(const MechParams& P, bool assume_2d, const double y[6],
                                               double l, double h, double eta0, double eta1_in,
                                               double ss, const EndPow& w, const Vel* __restrict__ drp,
                                               const double f[6], double v[6])
{
    const double R = P.R, E0 = P.E0, coul = P.coulomb;
    const double nx = y[3], ny = y[4], nz = y[5];
    const bool contacting = surface_contact(P, assume_2d, y, h);
    if (P.no_surface || !contacting || assume_2d)
        velocity_free_or_flat(P, contacting, y, l, eta0, eta1_in, drp, f, v);
    else
    {
        double eta1 = eta1_in;
        double A1, A2, A3;
        area_integrals(P, nz, h, ss, w, A1, A2, A3);
        if (coul > 0)
        {
            const double2 d01 = __ldg(reinterpret_cast<const double2*>(drp->v));
            const double2 d23 = __ldg(reinterpret_cast<const double2*>(drp->v) + 1);
            const double2 d45 = __ldg(reinterpret_cast<const double2*>(drp->v) + 2);
            double drxy = sqrt(d01.x * d01.x + d01.y * d01.y);
            double dnxy = sqrt(d23.y * d23.y + d45.x * d45.x);
            double friction_norm = (A1 * drxy + A2 * dnxy) * (eta1 / R);
            const double inz = 1.0 / nz;
            double max_norm = (1 - nz * nz) * integral1(w, inz, h, 4, ss)
                            + P.sqrtR * nz * nz * integral1(w, inz, h, 3, ss);
            max_norm *= (2 * E0 * coul);
            if (friction_norm > max_norm) eta1 = max_norm * R / (A1 * drxy + A2 * dnxy);
        }
        const double c1 = eta0 * l + (eta1 / R) * A1;
        const double c2 = eta0 * l;
        const double c4 = c2 * l * l / 12;
        const double c3 = c4 + (eta1 / R) * A3;
        const double c5 = (eta1 / R) * A2;
        const double ic1 = 1.0 / c1, ic4 = 1.0 / c4;
        const double c5c1 = c5 * ic1;
        const double term1 = c3 - c5 * c5c1;
        const double it1 = 1.0 / term1;
        const double w4 = f[3] - f[0] * c5c1;
        const double w5 = f[4] - f[1] * c5c1;
        const double nx2 = nx * it1, ny2 = ny * it1, nz2 = nz * ic4;
        const double alpha = 2 * ((nx * nx2 + ny * ny2) + nz * nz2);
        const double beta = -((w4 * nx2 + w5 * ny2) + f[5] * nz2);
        const double lambda = beta / alpha;
        v[5] = (f[5] + 2 * nz * lambda) * ic4;
        v[4] = (w5 + 2 * ny * lambda) * it1;
        v[3] = (w4 + 2 * nx * lambda) * it1;
        v[2] = f[2] / c2;
        v[1] = (f[1] - c5 * v[4]) * ic1;
        v[0] = (f[0] - c5 * v[3]) * ic1;
    }
}

// ---------------------------------------------------------------------------
// Mixed precision: the cell-surface forces, the area integrals and the velocity
// solve of a cell in surface contact (the third branch of getVelocities,
// mechanics.hpp:2191-2309, with mechanics.hpp:673-910 and integrals.hpp:116-463)
// in FP32.  R - rz, ss and the end overlaps are formed in FP64 before rounding, so
// shallow contacts keep their relative precision.  The overlap-power integrals over
// the contact come from the closed forms the FP64 path uses, except when both ends
// touch and the overlap varies by less than half its mid value along the cell
// (ss > 2h, i.e. rho = h nz / (R - rz) < 1/2): there the closed forms cancel, the
// differences p^a - q^a and the first moments losing up to 1/rho^2 of their digits,
// while the integrand is smooth with its nearest singularity at least two
// half-lengths from the centre, so a 6-point Gauss-Legendre rule (nodes and weights
// of Abramowitz & Stegun, Table 25.4) meets FP32 rounding.
// ---------------------------------------------------------------------------
struct SurfIntsF {      // integrals over the contact, s in [-h, min(ss, h)]
    float i_m12, i_12, i_1, i_32, i_2, i_52;    // int phi^a ds, a = -1/2, 1/2, 1, 3/2, 2, 5/2
    float s_m12, s_12, s_1, s_32;               // int s phi^a ds, a = -1/2, 1/2, 1, 3/2
    float s2_12;                                // int s^2 phi^(1/2) ds
};

// phi^(e/2) from phi and its square root, e = 1..9
__device__ __forceinline__ float half_pow_f(float x, float sx, int e)
{
    float r = (e & 1) ? sx : 1.f;
    for (int k = 0; k < (e >> 1); ++k) r *= x;
    return r;
}

// integrals.hpp:116-140 (integral1) and :159-184 (integral2) in FP32, exponent e/2 - 1:
// both ends in contact when ss > h, the lower end only when -h < ss <= h
__device__ __forceinline__ float integral1_f(float p, float q, float sp, float sq, float inz, float h, int e,
                                             float ss)
{
    const float ig = 2.f / (float)e;
    if (ss > h) return (half_pow_f(p, sp, e) - half_pow_f(q, sq, e)) * inz * ig;
    return half_pow_f(p, sp, e) * inz * ig;
}
__device__ __forceinline__ float integral2_f(float p, float q, float sp, float sq, float inz, float h, int e,
                                             float ss)
{
    const float term1 = integral1_f(p, q, sp, sq, inz, h, e + 2, ss);
    const float term2 = (ss > h) ? -h * (half_pow_f(p, sp, e) + half_pow_f(q, sq, e)) : -h * half_pow_f(p, sp, e);
    return (term1 + term2) * inz * (2.f / (float)e);
}

__device__ __forceinline__ SurfIntsF surface_integrals_f(double Rmrz, double nz_d, double h_d, double ss_d)
{
    SurfIntsF I;
    const float h = (float)h_d, nz = (float)nz_d, ss = (float)ss_d;
    if (ss_d > 2 * h_d)
    {
        const float x[3] = {0.2386191860831969f, 0.6612093864662645f, 0.9324695142031521f};
        const float w[3] = {0.4679139345726910f, 0.3607615730481386f, 0.1713244923791704f};
        const float phi0 = (float)Rmrz, hn = h * nz;
        float a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, b0 = 0, b1 = 0, b2 = 0, b3 = 0, c1 = 0;
#pragma unroll
        for (int k = 0; k < 6; ++k)
        {
            const float xk = (k & 1) ? -x[k >> 1] : x[k >> 1];
            const float wk = w[k >> 1] * h;
            const float sk = h * xk;
            const float ph = phi0 - xk * hn;
            const float r = sqrtf(ph), ir = 1.f / r;
            const float ph32 = ph * r;
            a0 += wk * ir; a1 += wk * r; a2 += wk * ph; a3 += wk * ph32; a4 += wk * (ph * ph); a5 += wk * (ph * ph32);
            b0 += wk * sk * ir; b1 += wk * sk * r; b2 += wk * sk * ph; b3 += wk * sk * ph32;
            c1 += wk * sk * sk * r;
        }
        I.i_m12 = a0; I.i_12 = a1; I.i_1 = a2; I.i_32 = a3; I.i_2 = a4; I.i_52 = a5;
        I.s_m12 = b0; I.s_12 = b1; I.s_1 = b2; I.s_32 = b3; I.s2_12 = c1;
        return I;
    }
    // end overlaps in FP64 (integrals.hpp:56-60), then rounded
    const double pd = Rmrz - (-h_d) * nz_d, qd = (ss_d > h_d) ? Rmrz - h_d * nz_d : 0.0;
    const float p = (float)pd, q = (float)qd, sp = sqrtf(p), sq = sqrtf(q);
    const float inz = 1.f / nz;
    I.i_m12 = integral1_f(p, q, sp, sq, inz, h, 1, ss);
    I.i_12 = integral1_f(p, q, sp, sq, inz, h, 3, ss);
    I.i_1 = integral1_f(p, q, sp, sq, inz, h, 4, ss);
    I.i_32 = integral1_f(p, q, sp, sq, inz, h, 5, ss);
    I.i_2 = integral1_f(p, q, sp, sq, inz, h, 6, ss);
    I.i_52 = integral1_f(p, q, sp, sq, inz, h, 7, ss);
    I.s_m12 = integral2_f(p, q, sp, sq, inz, h, 1, ss);
    I.s_12 = integral2_f(p, q, sp, sq, inz, h, 3, ss);
    I.s_1 = integral2_f(p, q, sp, sq, inz, h, 4, ss);
    I.s_32 = integral2_f(p, q, sp, sq, inz, h, 5, ss);
    // integrals.hpp:400-463: int3 = (2 int2b + h^2 (p^(3/2) - q^(3/2))) / (1.5 nz)
    I.s2_12 = (2.f * I.s_32 + h * h * (half_pow_f(p, sp, 3) - half_pow_f(q, sq, 3))) * inz * (1.f / 1.5f);
    return I;
}

// v (6 components) of a cell in surface contact at state y (not on the substrate:
// nz >= nz_threshold), from f0 = -dE/dq of the pair forces plus noise
__device__ __forceinline__ void velocity_contact_f32(const MechParams& P, const double y[6], double l_d,
                                                     double h_d, double eta0_d, double eta1_d, double sigma0_d,
                                                     const Vel* __restrict__ drp, const double f0[6], double v[6])
{
    const double Rmrz = P.R - y[2];
    const double ss_d = Rmrz / y[5];
    const SurfIntsF I = surface_integrals_f(Rmrz, y[5], h_d, ss_d);
    const float R = (float)P.R, E0 = (float)P.E0, sqrtR = (float)P.sqrtR;
    const float nx = (float)y[3], ny = (float)y[4], nz = (float)y[5];
    const float h = (float)h_d, l = (float)l_d, ss = (float)ss_d, sigma0 = (float)sigma0_d;
    const float nz2 = nz * nz, onz = 1.f - nz2;
    const bool partial = fabs(ss_d) < h_d;
    const float i4 = (ss_d > h_d) ? 2.f * h : ss + h;                 // integral4 (ss > -h here)
    // cell-surface repulsion, mechanics.hpp:673-780
    const float pf0 = 2.f * E0, pf1 = (8.f / 3.f) * E0 * sqrtR, pf2 = 2.f * E0 * sqrtR;
    const float rep_n = onz * I.i_1 + sqrtR * nz2 * I.i_12;
    const float rep2 = -pf0 * rep_n;
    const float rep5 = -pf0 * nz * I.i_2 - pf0 * onz * I.s_1 + pf1 * nz * I.i_32 - pf2 * nz2 * I.s_12;
    // cell-surface adhesion, mechanics.hpp:800-910
    const float a0 = sqrtR / 2.f, a1 = 2.f * 3.14159265358979f * R, a2 = 2.f * sqrtR;
    const float adh2 = (a0 * onz * I.i_m12 + (partial ? (a1 / 2.f) * nz : 0.f)) * sigma0;
    const float adh5 = (a2 * nz * I.i_12 + a0 * onz * I.s_m12 - a1 * nz * i4
                        + (partial ? (a1 / 2.f) * (float)Rmrz : 0.f)) * sigma0;
    // area integrals, integrals.hpp:400-463
    const float piRnz2 = 3.14159265358979f * R * nz2;
    const float i5 = (ss_d <= h_d) ? (ss * ss - h * h) / 2.f : 0.f;
    const float i6 = (ss_d > h_d) ? 2.f * h * h * h / 3.f : (ss * ss * ss + h * h * h) / 3.f;
    const float A1 = sqrtR * onz * I.i_12 + piRnz2 * i4;
    const float A2 = sqrtR * onz * I.s_12 + piRnz2 * i5;
    const float A3 = sqrtR * onz * I.s2_12 + piRnz2 * i6;
    // generalised forces in FP64, then the solve (mechanics.hpp:2191-2309) in FP32
    const float f0f = (float)f0[0], f1f = (float)f0[1], f3f = (float)f0[3], f4f = (float)f0[4];
    const float f2f = (float)((f0[2] - (double)rep2) - (double)adh2);
    const float f5f = (float)((f0[5] - (double)rep5) - (double)adh5);
    float eta1 = (float)eta1_d;
    const float coul = (float)P.coulomb;
    if (coul > 0.f)
    {
        const double2 d01 = __ldg(reinterpret_cast<const double2*>(drp->v));
        const double2 d23 = __ldg(reinterpret_cast<const double2*>(drp->v) + 1);
        const double2 d45 = __ldg(reinterpret_cast<const double2*>(drp->v) + 2);
        const float drxy = sqrtf((float)(d01.x * d01.x + d01.y * d01.y));
        const float dnxy = sqrtf((float)(d23.y * d23.y + d45.x * d45.x));
        const float friction_norm = (A1 * drxy + A2 * dnxy) * (eta1 / R);
        const float max_norm = rep_n * (2.f * E0 * coul);
        if (friction_norm > max_norm) eta1 = max_norm * R / (A1 * drxy + A2 * dnxy);
    }
    const float eR = eta1 / R;
    const float c2 = (float)eta0_d * l;
    const float c1 = c2 + eR * A1;
    const float c4 = c2 * l * l / 12.f;
    const float c3 = c4 + eR * A3;
    const float c5 = eR * A2;
    const float ic1 = 1.f / c1, ic4 = 1.f / c4;
    const float c5c1 = c5 * ic1;
    const float it1 = 1.f / (c3 - c5 * c5c1);
    const float w4 = f3f - f0f * c5c1;
    const float w5 = f4f - f1f * c5c1;
    const float nx2 = nx * it1, ny2 = ny * it1, nzc = nz * ic4;
    const float alpha = 2.f * ((nx * nx2 + ny * ny2) + nz * nzc);
    const float beta = -((w4 * nx2 + w5 * ny2) + f5f * nzc);
    const float lambda = beta / alpha;
    const float v4 = (w5 + 2.f * ny * lambda) * it1;
    const float v3 = (w4 + 2.f * nx * lambda) * it1;
    v[5] = (double)((f5f + 2.f * nz * lambda) * ic4);
    v[4] = (double)v4;
    v[3] = (double)v3;
    v[2] = (double)(f2f / c2);
    v[1] = (double)((f1f - c5 * v4) * ic1);
    v[0] = (double)((f0f - c5 * v3) * ic1);
}

}   // namespace abm
