// ORACLE — test infrastructure only.  A plain C++17 restatement of the 3-D
// mechanics step of kmnam/biofilm-ABMs (ABM-3d/ABM-3d-cpp), against which tests/ and
// __graft_entry__.smoke() compare the CUDA path, and which bench.py's CPU baseline leg
// times.  The product library never links, includes or calls anything under oracle/.
// Beyond the adaptive Runge-Kutta loop it restates, for the steps next to that path:
// cell-cell kinetic friction, the velocity-Verlet integrator with the constrained force
// forms, phenotype switching with its ramps, local viscosity and basal-only compaction,
// the variable-gamma JKR table, and the JKR equilibrium solves for gamma from eqdist.
//
// Every function names the reference file:line it restates.  The reference
// itself cannot be compiled here (Eigen, Boost and CGAL are absent), so:
//   * CGAL's Segment_3/Segment_3 squared_distance (distances.hpp:341) is
//     replaced by Ericson's clamped closest-point method for two segments
//     (C. Ericson, Real-Time Collision Detection, 2005, sec. 5.1.9), which
//     returns the same unique minimiser for non-parallel segments; it is pinned
//     against the reference's own known-answer cases (testDistBetweenCells.cpp).
//   * the MPFR Aberth quartic solve for the JKR radius table (jkr.hpp:67-144)
//     is replaced by a bracketed Newton solve of the same quartic in long
//     double, pinned by the invariants of testJKR.cpp:26-83.
//   * boost::random::mt19937 draws are replaced by the counter-based Philox
//     policy of philox.hpp (no reference test pins the mt19937 stream).
// Arrays are column-major (n rows x ncols), exactly like the reference's
// Eigen::Array<double, Dynamic, Dynamic>, so a reference cell array can be
// handed in unchanged.  Vector sums are evaluated as ((x + y) + z) and the
// file is compiled with -ffp-contract=off.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <random>
#include <stdexcept>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "philox.hpp"
#include "detmath.hpp"

namespace oracle {

// ABM-3d/ABM-3d-cpp/include/indices.hpp:17-47 ; gamma column simulation.hpp:1180
enum Col3 {
    C_ID = 0, C_RX = 1, C_RY = 2, C_RZ = 3, C_NX = 4, C_NY = 5, C_NZ = 6,
    C_DRX = 7, C_DRY = 8, C_DRZ = 9, C_DNX = 10, C_DNY = 11, C_DNZ = 12,
    C_L = 13, C_HALF_L = 14, C_T0 = 15, C_GROWTH = 16, C_ETA0 = 17,
    C_ETA1 = 18, C_SIGMA0 = 19, C_GROUP = 20, C_GAMMA = 21
};
const int NCOLS_REQUIRED_3D = 21;
const double PI = 3.141592653589793238462643383279502884;
const double TWO_PI = 6.283185307179586476925286766559005768;

struct Cells {
    int n = 0, ncols = 0;
    std::vector<double> a;   // column-major, leading dimension n
    Cells() {}
    Cells(int n_, int ncols_) : n(n_), ncols(ncols_), a((size_t)n_ * ncols_, 0.0) {}
    double& operator()(int i, int j) { return a[(size_t)j * n + i]; }
    double operator()(int i, int j) const { return a[(size_t)j * n + i]; }
};

struct V3 { double x, y, z; };
inline V3 v3(double x, double y, double z) { V3 v = {x, y, z}; return v; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(double s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double norm(V3 a) { return std::sqrt((a.x * a.x + a.y * a.y) + a.z * a.z); }

inline V3 cell_r(const Cells& c, int i) { return v3(c(i, C_RX), c(i, C_RY), c(i, C_RZ)); }
inline V3 cell_n(const Cells& c, int i) { return v3(c(i, C_NX), c(i, C_NY), c(i, C_NZ)); }

// ------------------------------------------------------------------------
// Segment distance (ABM-3d/ABM-3d-cpp/include/distances.hpp)
// ------------------------------------------------------------------------

// distances.hpp:92-105
inline double nearest_body_coord(V3 r, V3 n, double half_l, V3 q)
{
    double s = dot(q - r, n);
    if (std::fabs(s) <= half_l) return s;
    else if (s > half_l) return half_l;
    else return -half_l;
}

inline double clamp01(double x) { return x < 0 ? 0 : (x > 1 ? 1 : x); }

// Stand-in for CGAL::Distance_3::internal::squared_distance(Segment_3, Segment_3)
// (distances.hpp:341): returns the parameters (x, y) in [0, 1] of the closest
// points p1 + x (q1 - p1) and p2 + y (q2 - p2).  Method: Ericson, Real-Time
// Collision Detection (2005), sec. 5.1.9, "ClosestPtSegmentSegment".
inline void closest_params_segments(V3 p1, V3 q1, V3 p2, V3 q2, double& x, double& y)
{
    V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    if (a <= 0 && e <= 0) { x = 0; y = 0; return; }
    if (a <= 0) { x = 0; y = clamp01(f / e); return; }
    double c = dot(d1, r);
    if (e <= 0) { y = 0; x = clamp01(-c / a); return; }
    double b = dot(d1, d2);
    double denom = a * e - b * b;
    double s = (denom != 0) ? clamp01((b * f - c * e) / denom) : 0.0;
    double t = (b * s + f) / e;
    if (t < 0) { t = 0; s = clamp01(-c / a); }
    else if (t > 1) { t = 1; s = clamp01((b - c) / a); }
    x = s; y = t;
}

struct DistResult { V3 d; double s, t; };

// distances.hpp:206-357 (distBetweenCells); segment endpoints as in
// generateSegments (distances.hpp:59-80)
inline DistResult dist_between_cells(V3 r1, V3 n1, double half_l1, V3 r2, V3 n2, double half_l2)
{
    DistResult out;
    out.d = v3(0, 0, 0); out.s = 0; out.t = 0;
    double cos_theta = dot(n1, n2);
    if (cos_theta >= 0.9999 || cos_theta <= -0.9999)
    {
        V3 p1 = r1 - half_l1 * n1, q1 = r1 + half_l1 * n1;
        V3 p2 = r2 - half_l2 * n2, q2 = r2 + half_l2 * n2;
        double s_p1 = nearest_body_coord(r2, n2, half_l2, p1);
        double s_q1 = nearest_body_coord(r2, n2, half_l2, q1);
        V3 d_p1 = (r2 + s_p1 * n2) - p1;
        V3 d_q1 = (r2 + s_q1 * n2) - q1;
        double dist_p1 = norm(d_p1), dist_q1 = norm(d_q1);
        if (s_p1 == s_q1)
        {
            if (dist_p1 < dist_q1) { out.s = -half_l1; out.t = s_p1; out.d = d_p1; }
            else { out.s = half_l1; out.t = s_q1; out.d = d_q1; }
        }
        else
        {
            double s_p2 = nearest_body_coord(r1, n1, half_l1, p2);
            double s_q2 = nearest_body_coord(r1, n1, half_l1, q2);
            V3 d_p2 = (r1 + s_p2 * n1) - p2;
            V3 d_q2 = (r1 + s_q2 * n1) - q2;
            double dist_p2 = norm(d_p2), dist_q2 = norm(d_q2);
            // std::sort of four (dist, idx) pairs by dist (distances.hpp:274-286):
            // libstdc++ sorts a 4-element range by insertion sort, which keeps
            // ties in their original order, so a stable insertion sort is used.
            double dv[4] = {dist_p1, dist_q1, dist_p2, dist_q2};
            int iv[4] = {0, 1, 2, 3};
            for (int a = 1; a < 4; ++a)
            {
                double kd = dv[a]; int ki = iv[a]; int b = a - 1;
                while (b >= 0 && kd < dv[b]) { dv[b + 1] = dv[b]; iv[b + 1] = iv[b]; --b; }
                dv[b + 1] = kd; iv[b + 1] = ki;
            }
            bool m0 = (iv[0] == 0 || iv[1] == 0), m1 = (iv[0] == 1 || iv[1] == 1);
            bool m2 = (iv[0] == 2 || iv[1] == 2);
            if (m0)
            {
                if (m1)
                {
                    out.s = 0.0;
                    out.t = nearest_body_coord(r2, n2, half_l2, r1);
                    out.d = (r2 + out.t * n2) - r1;
                }
                else if (m2)
                {
                    out.s = (-half_l1 + s_p2) / 2;
                    out.t = nearest_body_coord(r2, n2, half_l2, r1 + out.s * n1);
                    out.d = ((r2 + out.t * n2) - r1) - out.s * n1;
                }
                else
                {
                    out.s = (-half_l1 + s_q2) / 2;
                    out.t = nearest_body_coord(r2, n2, half_l2, r1 + out.s * n1);
                    out.d = ((r2 + out.t * n2) - r1) - out.s * n1;
                }
            }
            else if (m1)
            {
                if (m2)
                {
                    out.s = (half_l1 + s_p2) / 2;
                    out.t = nearest_body_coord(r2, n2, half_l2, r1 + out.s * n1);
                    out.d = ((r2 + out.t * n2) - r1) - out.s * n1;
                }
                else
                {
                    out.s = (half_l1 + s_q2) / 2;
                    out.t = nearest_body_coord(r2, n2, half_l2, r1 + out.s * n1);
                    out.d = ((r2 + out.t * n2) - r1) - out.s * n1;
                }
            }
            else
            {
                out.t = 0.0;
                out.s = nearest_body_coord(r1, n1, half_l1, r2);
                out.d = (r2 - r1) - out.s * n1;
            }
        }
    }
    else
    {
        V3 p1 = r1 - half_l1 * n1, q1 = r1 + half_l1 * n1;
        V3 p2 = r2 - half_l2 * n2, q2 = r2 + half_l2 * n2;
        double x, y;
        closest_params_segments(p1, q1, p2, q2, x, y);
        out.s = x * 2 * half_l1 - half_l1;
        out.t = y * 2 * half_l2 - half_l2;
        out.d = ((r2 + out.t * n2) - r1) - out.s * n1;
    }
    return out;
}

inline DistResult dist_cells(const Cells& c, int i, int j)
{
    return dist_between_cells(cell_r(c, i), cell_n(c, i), c(i, C_HALF_L),
                              cell_r(c, j), cell_n(c, j), c(j, C_HALF_L));
}

// ------------------------------------------------------------------------
// Neighbor table (mechanics.hpp:520-648).  Row = (i, j, dx, dy, dz, si, sj)
// ------------------------------------------------------------------------
struct Neighbors {
    std::vector<int> i, j;
    std::vector<double> dx, dy, dz, si, sj;
    int size() const { return (int)i.size(); }
};

// mechanics.hpp:520-593 (getCellNeighbors): O(n^2), rows i-major, j < i ascending
inline Neighbors get_cell_neighbors(const Cells& cells, double neighbor_threshold,
                                    double R, double Ldiv)
{
    Neighbors nb;
    int n = cells.n;
    if (n == 1) return nb;
    const double prefilter = neighbor_threshold + Ldiv + 2 * R;
    for (int i = 0; i < n; ++i)
    {
        V3 ri = cell_r(cells, i);
        for (int j = 0; j < i; ++j)
        {
            double dist_rij = norm(ri - cell_r(cells, j));
            if (dist_rij < prefilter)
            {
                DistResult res = dist_cells(cells, i, j);
                if (norm(res.d) < neighbor_threshold)
                {
                    nb.i.push_back(i); nb.j.push_back(j);
                    nb.dx.push_back(res.d.x); nb.dy.push_back(res.d.y); nb.dz.push_back(res.d.z);
                    nb.si.push_back(res.s); nb.sj.push_back(res.t);
                }
            }
        }
    }
    return nb;
}

// The same table as get_cell_neighbors from a uniform grid of bins no smaller than the
// prefilter radius, so that every pair that passes the prefilter lies in adjacent bins:
// each cell's row is made from the cells of its 27 surrounding bins (OpenMP over the
// rows), with the same prefilter and distance arithmetic on (i, j), and sorted by j.
// Not the reference's procedure: the "optimized CPU" figure reported beside the
// reference-faithful CPU run uses it (with cpu_optimized in the parameters).
inline Neighbors get_cell_neighbors_grid(const Cells& cells, double neighbor_threshold, double R, double Ldiv)
{
    Neighbors nb;
    const int n = cells.n;
    if (n <= 1) return nb;
    const double prefilter = neighbor_threshold + Ldiv + 2 * R;
    double lo[3] = {cells(0, C_RX), cells(0, C_RY), cells(0, C_RZ)}, hi[3] = {lo[0], lo[1], lo[2]};
    for (int i = 1; i < n; ++i)
    {
        const double r[3] = {cells(i, C_RX), cells(i, C_RY), cells(i, C_RZ)};
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], r[a]); hi[a] = std::max(hi[a], r[a]); }
    }
    // bins of edge >= prefilter, at most about 4 n of them (a sparse state widens the edge)
    double edge = prefilter;
    long long dims[3];
    for (;;)
    {
        long long total = 1;
        for (int a = 0; a < 3; ++a)
        {
            dims[a] = (long long)std::floor((hi[a] - lo[a]) / edge) + 1;
            total *= dims[a];
        }
        if (total <= 4LL * n + 64) break;
        edge *= 2;
    }
    auto bin_of = [&](int i, long long b[3]) {
        const double r[3] = {cells(i, C_RX), cells(i, C_RY), cells(i, C_RZ)};
        for (int a = 0; a < 3; ++a)
            b[a] = std::min(dims[a] - 1, std::max(0LL, (long long)std::floor((r[a] - lo[a]) / edge)));
    };
    const long long nbins = dims[0] * dims[1] * dims[2];
    std::vector<int> start((size_t)nbins + 1, 0), members((size_t)n);
    std::vector<long long> key((size_t)n);
    for (int i = 0; i < n; ++i)
    {
        long long b[3];
        bin_of(i, b);
        key[i] = (b[2] * dims[1] + b[1]) * dims[0] + b[0];
        ++start[key[i] + 1];
    }
    for (long long b = 0; b < nbins; ++b) start[b + 1] += start[b];
    {
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (int i = 0; i < n; ++i) members[fill[key[i]]++] = i;
    }
    struct Row { int j; DistResult res; };
    std::vector<std::vector<Row> > rows((size_t)n);
    #pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i)
    {
        long long b[3];
        bin_of(i, b);
        const V3 ri = cell_r(cells, i);
        std::vector<Row>& out = rows[i];
        for (long long z = std::max(0LL, b[2] - 1); z <= std::min(dims[2] - 1, b[2] + 1); ++z)
            for (long long y = std::max(0LL, b[1] - 1); y <= std::min(dims[1] - 1, b[1] + 1); ++y)
                for (long long x = std::max(0LL, b[0] - 1); x <= std::min(dims[0] - 1, b[0] + 1); ++x)
                {
                    const long long bb = (z * dims[1] + y) * dims[0] + x;
                    for (int q = start[bb]; q < start[bb + 1]; ++q)
                    {
                        const int j = members[q];
                        if (j >= i || !(norm(ri - cell_r(cells, j)) < prefilter)) continue;
                        const DistResult res = dist_cells(cells, i, j);
                        if (norm(res.d) < neighbor_threshold) out.push_back(Row{j, res});
                    }
                }
        std::sort(out.begin(), out.end(), [](const Row& a, const Row& c) { return a.j < c.j; });
    }
    for (int i = 0; i < n; ++i)
        for (const Row& r : rows[i])
        {
            nb.i.push_back(i); nb.j.push_back(r.j);
            nb.dx.push_back(r.res.d.x); nb.dy.push_back(r.res.d.y); nb.dz.push_back(r.res.d.z);
            nb.si.push_back(r.res.s); nb.sj.push_back(r.res.t);
        }
    return nb;
}

// mechanics.hpp:604-648 (updateNeighborDistances)
inline void update_neighbor_distances(const Cells& cells, Neighbors& nb)
{
    for (int k = 0; k < nb.size(); ++k)
    {
        DistResult res = dist_cells(cells, nb.i[k], nb.j[k]);
        nb.dx[k] = res.d.x; nb.dy[k] = res.d.y; nb.dz[k] = res.d.z;
        nb.si[k] = res.s; nb.sj[k] = res.t;
    }
}

// ------------------------------------------------------------------------
// Auxiliary integrals (ABM-3d/ABM-3d-cpp/include/integrals.hpp)
// ------------------------------------------------------------------------
inline double sstar(double rz, double nz, double R) { return (R - rz) / nz; }        // :35-45
// x^e for the integrals' exponents gamma + 1: x * x for the square, the C library for the
// others.  g++ folds pow(x, 2.0) into x * x only where inlining makes the exponent a
// constant, and the C library's pow may differ from x * x in the last bit, so the square is
// written out: the last bit of an integral then does not depend on which calls the compiler
// inlines (an unrelated edit once moved one cell's velocity by two ulps that way).
inline double pow_e(double x, double e) { return e == 2.0 ? x * x : std::pow(x, e); }
inline double phi(double rz, double nz, double R, double s) { return R - rz - s * nz; }  // :56-60

// integrals.hpp:116-140
inline double integral1(double rz, double nz, double R, double half_l, double gamma, double ss)
{
    if (ss > half_l)
    {
        double o1 = pow_e(phi(rz, nz, R, -half_l), gamma + 1);
        double o2 = pow_e(phi(rz, nz, R, half_l), gamma + 1);
        return (o1 - o2) / (nz * (gamma + 1));
    }
    else if (ss > -half_l)
    {
        double o1 = pow_e(phi(rz, nz, R, -half_l), gamma + 1);
        return o1 / (nz * (gamma + 1));
    }
    return 0;
}

// integrals.hpp:159-184
inline double integral2(double rz, double nz, double R, double half_l, double gamma, double ss)
{
    double term1 = integral1(rz, nz, R, half_l, gamma + 1, ss);
    double term2 = 0;
    if (ss > half_l)
    {
        double o1 = pow_e(phi(rz, nz, R, -half_l), gamma + 1);
        double o2 = pow_e(phi(rz, nz, R, half_l), gamma + 1);
        term2 = -half_l * (o1 + o2);
    }
    else if (ss > -half_l)
    {
        double o1 = pow_e(phi(rz, nz, R, -half_l), gamma + 1);
        term2 = -half_l * o1;
    }
    return (term1 + term2) / (nz * (gamma + 1));
}

// integrals.hpp:250-266
inline double integral4(double nz, double half_l, double ss)
{
    (void)nz;
    if (ss > half_l) return 2 * half_l;
    else if (ss > -half_l) return ss + half_l;
    return 0;
}
// integrals.hpp:279-291
inline double integral5(double nz, double half_l, double ss)
{
    (void)nz;
    if (-half_l < ss && ss <= half_l) return (ss * ss - half_l * half_l) / 2.0;
    return 0.0;
}
// integrals.hpp:304-318
inline double integral6(double nz, double half_l, double ss)
{
    (void)nz;
    if (ss > half_l) return 2 * half_l * half_l * half_l / 3.0;
    else if (ss > -half_l) return (ss * ss * ss + half_l * half_l * half_l) / 3.0;
    return 0.0;
}

// integrals.hpp:400-463 (areaIntegrals)
inline void area_integrals(double rz, double nz, double R, double half_l, double ss,
                           double& area1, double& area2, double& area3)
{
    double int4 = integral4(nz, half_l, ss);
    double int5 = integral5(nz, half_l, ss);
    double int6 = integral6(nz, half_l, ss);
    double int1a = integral1(rz, nz, R, half_l, 0.5, ss);
    double int1b = integral1(rz, nz, R, half_l, 1.5, ss);
    double int1c = integral1(rz, nz, R, half_l, 2.5, ss);
    double term1 = std::sqrt(R) * (1 - nz * nz) * int1a;
    double term2 = PI * R * nz * nz * int4;
    area1 = term1 + term2;
    double overlap1 = 0, overlap2 = 0;
    if (ss > half_l) { overlap1 = phi(rz, nz, R, -half_l); overlap2 = phi(rz, nz, R, half_l); }
    else if (ss > -half_l) { overlap1 = phi(rz, nz, R, -half_l); }
    double o1p1 = std::pow(overlap1, 1.5), o2p1 = std::pow(overlap2, 1.5);
    term2 = -half_l * (o1p1 + o2p1);
    double int2a = (int1b + term2) / (1.5 * nz);
    term1 = std::sqrt(R) * (1 - nz * nz) * int2a;
    term2 = PI * R * nz * nz * int5;
    area2 = term1 + term2;
    double o1p2 = o1p1 * overlap1, o2p2 = o2p1 * overlap2;
    term2 = -half_l * (o1p2 + o2p2);
    double int2b = (int1c + term2) / (2.5 * nz);
    term1 = 2 * int2b;
    term2 = half_l * half_l * (o1p1 - o2p1);
    double int3 = (term1 + term2) / (1.5 * nz);
    term1 = std::sqrt(R) * (1 - nz * nz) * int3;
    term2 = PI * R * nz * nz * int6;
    area3 = term1 + term2;
}

// ------------------------------------------------------------------------
// JKR radius table and lookup
// ------------------------------------------------------------------------

// Eigen::Matrix::LinSpaced(n, low, high) for a real scalar with |high| >= |low|:
// low + i * step for i < n - 1 and exactly high at the last entry.
inline std::vector<double> linspaced(int n, double low, double high)
{
    std::vector<double> v(n);
    if (n == 1) { v[0] = high; return v; }
    double step = (high - low) / double(n - 1);
    for (int i = 0; i < n; ++i) v[i] = (i == n - 1) ? high : low + double(i) * step;
    return v;
}

// jkr.hpp:67-144 (jkrContactRadius(delta, Req, E, gamma).second): the larger
// positive real root a of  a^4 - 2 Req delta a^2 - (4 pi gamma Req^2 / E) a
// + delta^2 Req^2 = 0, i.e. the root of  g(a) = a^2/Req - 2 sqrt(pi gamma a/E)
// - delta  on the branch where g increases.  Solved in long double by
// bracketing plus Newton steps (the reference uses 100-digit MPFR Aberth).
inline double jkr_contact_radius(double delta, double Req, double E, double gamma)
{
    typedef long double LD;
    LD d = delta, R = Req, Ee = E, g = gamma, pi = 3.141592653589793238462643383279502884L;
    if (g <= 0) return (double)std::sqrt(R * d);
    // g(a) = a^2/R - 2 sqrt(pi g a / E) - d, minimum at a_min where g'(a) = 0
    auto G = [&](LD a) { return a * a / R - 2 * std::sqrt(pi * g * a / Ee) - d; };
    auto dG = [&](LD a) { return 2 * a / R - std::sqrt(pi * g / (Ee * a)); };
    LD a_min = std::cbrt(R * R * pi * g / (4 * Ee));
    LD lo = a_min, hi = std::max(a_min * 2, std::sqrt(R * std::max(d, (LD)0)) + a_min * 4 + 1e-6L);
    while (G(hi) < 0) hi *= 2;
    LD a = hi;
    for (int it = 0; it < 200; ++it)
    {
        LD ga = G(a);
        if (ga > 0) hi = a; else lo = a;
        LD step = ga / dG(a);
        LD an = a - step;
        if (!(an > lo && an < hi)) an = (lo + hi) / 2;
        if (std::fabs(an - a) <= 1e-19L * std::fabs(a)) { a = an; break; }
        a = an;
    }
    return (double)a;
}

// simulation.hpp:86-104 (calculateJKRContactRadii) over the overlap mesh of
// simulation.hpp:1379-1382
inline std::vector<double> jkr_radius_table(const std::vector<double>& overlaps, double gamma,
                                            double R, double E0)
{
    std::vector<double> radii(overlaps.size());
    for (size_t i = 0; i < overlaps.size(); ++i)
        radii[i] = jkr_contact_radius(overlaps[i], R / 2, E0, gamma);
    return radii;
}

// rootFinding.hpp:42-75 (newtonRaphson): Newton steps with a central-difference
// derivative of step dx until |f(x)| <= tol or max_iter steps; returns (x, f(x)).
template <typename F>
inline std::pair<double, double> newton_raphson(F func, double x0, double dx, double tol, int max_iter)
{
    double x = x0, fx = func(x);
    int iter = 0;
    while (std::fabs(fx) > tol && iter < max_iter)
    {
        double deriv = (func(x + dx) - func(x - dx)) / (2 * dx);
        x += -fx / deriv;
        fx = func(x);
        ++iter;
    }
    return std::make_pair(x, fx);
}

// jkr.hpp:1311-1339 (jkrEquilibriumDistance): the overlap where the JKR force
// (4/3) (E0/Req) a^3 - 4 sqrt(pi gamma E0) a^(3/2) vanishes, a the contact radius at
// that overlap, found by newtonRaphson from 2R - dinit and capped at 2R - dmin.
inline double jkr_equilibrium_distance(double R, double E0, double gamma, double dinit, double dmin,
                                       double increment_overlap, double newton_tol, int max_iter)
{
    const double Req = R / 2;
    auto force = [&](double x) {
        double a = jkr_contact_radius(x, Req, E0, gamma);
        return (4.0 / 3.0) * E0 / Req * a * a * a - 4 * std::sqrt(PI * gamma * E0) * std::pow(a, 1.5);
    };
    std::pair<double, double> res = newton_raphson(force, 2 * R - dinit, increment_overlap, newton_tol, max_iter);
    return 2 * R - std::min(res.first, 2 * R - dmin);
}

// jkr.hpp:1369-1407 (jkrOptimalSurfaceEnergyDensity) with the arguments of
// simulation.hpp:1355-1358: newtonRaphson on log10(gamma) from log10(100), step 1e-6,
// tolerance 1e-8 on the equilibrium distance, inner solves from dinit = 1.5 R with
// dmin = 2 Rcell, step 1e-8 and tolerance 1e-8, at most 1000 steps each.
inline double jkr_optimal_gamma(double R, double Rcell, double E0, double deq_target)
{
    auto func = [&](double x) {
        double gamma = std::pow(10.0, x);
        return jkr_equilibrium_distance(R, E0, gamma, 0.75 * 2 * R, 2 * Rcell, 1e-8, 1e-8, 1000) - deq_target;
    };
    return std::pow(10.0, newton_raphson(func, std::log10(100.0), 1e-6, 1e-8, 1000).first);
}

// utils.hpp:1169-1215 (nearestValue)
inline int nearest_value(const std::vector<double>& values, double x)
{
    int sz = (int)values.size();
    if (x <= values[0]) return 0;
    else if (x >= values[sz - 1]) return sz - 1;
    int low = 0, high = sz - 1, nearest_idx = 0;
    while (low <= high)
    {
        int mid = (low + high) / 2;
        if (values[mid] <= x && x < values[mid + 1]) { nearest_idx = mid; break; }
        else if (x >= values[mid + 1]) low = mid + 1;
        else high = mid - 1;
    }
    if (low > high) throw std::runtime_error("Unexpected error during binary search");
    if (x - values[nearest_idx] < values[nearest_idx + 1] - x) return nearest_idx;
    return nearest_idx + 1;
}

// ------------------------------------------------------------------------
// Parameters
// ------------------------------------------------------------------------
struct RngStream;

struct Params3 {
    double R = 0.8, Rcell = 0.5, E0 = 3900.0, Ecell = 3.9e6;
    double L0 = 2.0, Ldiv = 5.6;
    double neighbor_threshold = 3.6, nz_threshold = 1e-8;
    int adhesion_mode = 1;            // 0 none, 1 isotropic JKR with a fixed-gamma radius table
    int integration_mode = 1;         // 1 HE21, 2 BS32, 3 RKF45, 4 DP54 (simulation.hpp:45-55)
    double max_stepsize = 1e-6, min_stepsize = 1e-9;
    double max_error_allowed = 1e-8, min_error = 1e-30;
    int max_tries_update_stepsize = 3;
    int iter_update_stepsize = 1, iter_update_neighbors = 100;
    double max_rxy_noise = 0, max_rz_noise = 0, max_nxy_noise = 0, max_nz_noise = 0;
    double cell_surface_coulomb_coeff = 1.0;
    int no_surface = 0;
    double growth_mean = 0, growth_std = 0, daughter_length_std = 0;
    double daughter_angle_xy_bound = 0, daughter_angle_z_bound = 0;
    uint64_t rng_seed = 42;
    int n_start_multithread = 50;
    std::vector<double> jkr_overlaps, jkr_radii;
    // step-size controller: 0 the reference rule (simulation.hpp:1688-1769); 2 the PI
    // controller: every iteration's first attempt runs at a proposed dt and is accepted
    // as is when its scaled error E passes (E <= 1), otherwise the reference rule
    // continues from it; after each accepted step the next dt is the PI proposal
    // dt 0.9 E_n^(-0.7/k) E_(n-1)^(0.4/k), k = error order + 1, the factor held to
    // [0.2, 10] and dt to [min_stepsize, max_stepsize] (Gustafsson's PI rule with the
    // parameters of Hairer & Wanner, Solving ODEs II, sec. IV.2)
    int controller = 0;
    int friction_mode = 0;                 // FrictionMode: 0 NONE, 1 KINETIC (mechanics.hpp:61-65)
    double cell_cell_coulomb_coeff = 1.0;  // runSimulation's default (simulation.hpp:1162)
    double M0 = 0;                         // cell mass at length L0 (velocity Verlet)
    // phenotype switching and its ramps (switch.hpp:26-144; simulation.hpp:1340-1371,
    // 1650-1656, 1866-2022), two groups; basal-only compaction (simulation.hpp:1831-1856)
    int switch_mode = 0;                   // SwitchMode: 0 NONE, 1 MARKOV, 2 INHERIT
    int n_cells_start_switch = 0;
    double switch_rates[4] = {0, 0, 0, 0}; // 2 x 2, row = current group: rates (MARKOV) or probabilities (INHERIT)
    double group_growth_mean[2] = {0, 0}, group_growth_std[2] = {0, 0};   // per group, with switching on
    int n_attributes = 0;
    int attr_col[4] = {0, 0, 0, 0};
    double attr_target[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    double switch_timescale = 0;
    double max_gamma = 0;
    int modulate_local_viscosity = 0;
    double viscosity_lims[4] = {0, 0, 0, 0};   // 2 x 2: (min, max) per group
    int max_coordination_number = 1;
    int basal_only = 0;
    double basal_min_overlap = 0;
    // variable-gamma JKR table (IsotropicJKRDataVariableGamma, mechanics.hpp:159-199): radii on the
    // overlap mesh jkr_overlaps x the gamma mesh jkr_gammas, overlap-major; used when non-empty
    std::vector<double> jkr_gammas, jkr_radii2;
    // not the reference's procedure: the "optimized CPU" context figure (cell-list neighbor
    // build, pair forces with OpenMP over the pairs); off for every parity comparison
    int cpu_optimized = 0;
    // Random draws: the counter-based Philox policy (null, the default, which the CUDA path
    // shares), or one sequential stream drawn in the reference's order (a semantics check).
    RngStream* stream = nullptr;
    // divideCells of the 2-D model (2D/include/growth.hpp:252-258) draws one angle per daughter,
    // in the plane; with planar_division the restatement draws no out-of-plane angles (their
    // bound is 0 there, so only the stream's order changes)
    int planar_division = 0;
};

// The reference's random source (simulation.hpp:1173, 1298): one mt19937 (Matsumoto and
// Nishimura 1998) seeded with rng_seed, read through boost::random::uniform_01<>, which
// scales a 32-bit output x to x / 2^32.  Every draw of the loop comes from it in the
// reference's order: per try of divideCells the four daughter angles of each mother,
// then each mother's length fraction (two uniforms, Box-Muller), then the growth rates
// of the mothers and of the daughters (two each) (growth.hpp:252-350); n x 6 noise
// uniforms, cell-major, per stepRungeKuttaAdaptive call (mechanics.hpp:2493-2509); one
// uniform per cell, and two more for a switched cell's growth rate, in Markov switching
// (switch.hpp:55-75), and per daughter pair one, then two more uniforms and a growth
// rate for a switch, in inherited switching (switch.hpp:107-135).  `draws` counts them.
struct RngStream {
    std::mt19937 engine;
    long long draws = 0;
    explicit RngStream(uint32_t seed) : engine(seed) {}
    double uniform01()
    {
        ++draws;
        return (double)engine() * (1.0 / 4294967296.0);
    }
};

// getCellNeighbors as the loop calls it: the reference's O(n^2) procedure, or the
// cell-list build with cpu_optimized (the same table)
inline Neighbors build_neighbors(const Cells& cells, const Params3& p)
{
    return p.cpu_optimized ? get_cell_neighbors_grid(cells, p.neighbor_threshold, p.R, p.Ldiv)
                           : get_cell_neighbors(cells, p.neighbor_threshold, p.R, p.Ldiv);
}

struct Tableau {
    int s = 0; double error_order = 0;
    std::vector<double> A, b, bs;   // A row-major s x s
    double a(int i, int j) const { return A[(size_t)i * s + j]; }
};

// simulation.hpp:1207-1268
inline Tableau make_tableau(int mode)
{
    Tableau t;
    if (mode == 1)
    {
        t.s = 2; t.A = {0, 0, 1, 0}; t.b = {0.5, 0.5}; t.bs = {1, 0}; t.error_order = 1;
    }
    else if (mode == 2)
    {
        t.s = 4;
        t.A = {0, 0, 0, 0,  1. / 2., 0, 0, 0,  0, 3. / 4., 0, 0,  2. / 9., 1. / 3., 4. / 9., 0};
        t.b = {2. / 9., 1. / 3., 4. / 9., 0};
        t.bs = {7. / 24., 1. / 4., 1. / 3., 1. / 8.};
        t.error_order = 2;
    }
    else if (mode == 3)
    {
        t.s = 6;
        t.A = {0, 0, 0, 0, 0, 0,
               1. / 4., 0, 0, 0, 0, 0,
               3. / 32., 9. / 32., 0, 0, 0, 0,
               1932. / 2197., -7200. / 2197., 7296. / 2197., 0, 0, 0,
               439. / 216., -8.0, 3680. / 513., -845. / 4104., 0, 0,
               -8. / 27., 2.0, -3544. / 2565., 1859. / 4104., -11. / 40., 0};
        t.b = {16. / 135., 0, 6656. / 12825., 28561. / 56430., -9. / 50., 2. / 55.};
        t.bs = {25. / 216., 0, 1408. / 2565., 2197. / 4104., -1. / 5., 0};
        t.error_order = 4;
    }
    else if (mode == 4)
    {
        t.s = 7;
        t.A = {0, 0, 0, 0, 0, 0, 0,
               1. / 5., 0, 0, 0, 0, 0, 0,
               3. / 40., 9. / 40., 0, 0, 0, 0, 0,
               44. / 45., -56. / 15., 32. / 9., 0, 0, 0, 0,
               19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729, 0, 0, 0,
               9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656., 0, 0,
               35. / 384., 0, 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84., 0};
        t.b = {35. / 384., 0, 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84., 0};
        t.bs = {5179. / 57600., 0, 7571. / 16695., 393. / 640., -92097. / 339200., 187. / 2100., 1. / 40.};
        t.error_order = 4;
    }
    else throw std::runtime_error("unsupported integration mode");
    return t;
}

// simulation.hpp:1270-1274
inline void repulsion_prefactors(const Params3& p, double pf[3])
{
    pf[0] = (4. / 3.) * p.E0 * std::sqrt(p.R / 2);
    pf[1] = (4. / 3.) * p.Ecell * std::sqrt(p.Rcell / 2);
    pf[2] = (4. / 3.) * p.E0 * std::sqrt(p.R / 2) * std::pow(2 * (p.R - p.Rcell), 1.5);
}

// ------------------------------------------------------------------------
// Generalised forces (mechanics.hpp)
// ------------------------------------------------------------------------
typedef std::vector<double> Arr6;   // n x 6, column-major (ld = n)
inline double& A6(Arr6& a, int n, int i, int k) { return a[(size_t)k * n + i]; }
inline double A6c(const Arr6& a, int n, int i, int k) { return a[(size_t)k * n + i]; }

inline V3 cross(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// adhesion.hpp:282-370 (forcesIsotropicJKRLagrange, interpolate = true) with
// max_overlap = 2 (R - Rcell); rows = cells i, j.  With `constraint` (include_constraint,
// the velocity-Verlet form) the orientation rows are s (-(n1 . -v) n1 - v) and
// t ((n2 . -v) n2 + v), as the reference writes them, not a cross product
// (adhesion.hpp:355-366).
inline void jkr_forces(V3 d12, double R, double E0, double gamma, double s, double t,
                       const std::vector<double>& tab_delta, const std::vector<double>& tab_radius,
                       double max_overlap, double out[2][6], bool constraint = false,
                       V3 n1 = V3{0, 0, 0}, V3 n2 = V3{0, 0, 0})
{
    for (int a = 0; a < 2; ++a) for (int k = 0; k < 6; ++k) out[a][k] = 0;
    double dist = norm(d12);
    if (dist < 2 * R)
    {
        V3 d12n = v3(d12.x / dist, d12.y / dist, d12.z / dist);
        double delta = 2 * R - dist;
        if (max_overlap >= 0 && delta > max_overlap) delta = max_overlap;
        int idx_d1 = nearest_value(tab_delta, delta);
        int idx_d2 = (tab_delta[idx_d1] < delta ? idx_d1 + 1 : idx_d1 - 1);
        if (idx_d1 > idx_d2) std::swap(idx_d1, idx_d2);
        double d1 = tab_delta[idx_d1], d2 = tab_delta[idx_d2];
        double r1 = tab_radius[idx_d1], r2 = tab_radius[idx_d2];
        double radius = (r1 * (d2 - delta) + r2 * (delta - d1)) / (d2 - d1);
        double Req = R / 2;
        double a3 = radius * radius * radius;
        double term1 = 4 * E0 * a3 / (3 * Req);
        double term2 = 4 * std::sqrt(PI * a3 * gamma * E0);
        V3 v = (term2 - term1) * d12n;
        out[0][0] = -v.x; out[0][1] = -v.y; out[0][2] = -v.z;
        out[1][0] = v.x; out[1][1] = v.y; out[1][2] = v.z;
        if (!constraint)
        {
            out[0][3] = -s * v.x; out[0][4] = -s * v.y; out[0][5] = -s * v.z;
            out[1][3] = t * v.x; out[1][4] = t * v.y; out[1][5] = t * v.z;
        }
        else
        {
            const V3 mv = v3(-v.x, -v.y, -v.z);
            const double w1 = dot(n1, mv), w2 = dot(n2, mv);
            const V3 a = (-w1) * n1 - v, b = w2 * n2 + v;
            out[0][3] = s * a.x; out[0][4] = s * a.y; out[0][5] = s * a.z;
            out[1][3] = t * b.x; out[1][4] = t * b.y; out[1][5] = t * b.z;
        }
    }
}

// adhesion.hpp:412-526 (forcesIsotropicJKRLagrange, variable gamma, interpolate = true): the
// contact radius interpolated bilinearly between the four table points around (delta, gamma),
// each neighbor chosen on the side of the value; then the forces of jkr_forces.
inline void jkr_forces_variable(V3 d12, double R, double E0, double gamma, double s, double t,
                                const std::vector<double>& tab_delta, const std::vector<double>& tab_gamma,
                                const std::vector<double>& tab_radius, double max_overlap, double out[2][6],
                                bool constraint = false, V3 n1 = V3{0, 0, 0}, V3 n2 = V3{0, 0, 0})
{
    for (int a = 0; a < 2; ++a) for (int k = 0; k < 6; ++k) out[a][k] = 0;
    const double dist = norm(d12);
    if (!(dist < 2 * R)) return;
    const V3 d12n = v3(d12.x / dist, d12.y / dist, d12.z / dist);
    double delta = 2 * R - dist;
    if (max_overlap >= 0 && delta > max_overlap) delta = max_overlap;
    int id1 = nearest_value(tab_delta, delta), ig1 = nearest_value(tab_gamma, gamma);
    int id2 = (tab_delta[id1] < delta ? id1 + 1 : id1 - 1);
    if (id1 > id2) std::swap(id1, id2);
    int ig2 = (tab_gamma[ig1] < gamma ? ig1 + 1 : ig1 - 1);
    if (ig1 > ig2) std::swap(ig1, ig2);
    const size_t ng = tab_gamma.size();
    const double d1 = tab_delta[id1], d2 = tab_delta[id2], g1 = tab_gamma[ig1], g2 = tab_gamma[ig2];
    const double denom = (d2 - d1) * (g2 - g1);
    const double w11 = (d2 - delta) * (g2 - gamma) / denom;
    const double w12 = (d2 - delta) * (gamma - g1) / denom;
    const double w21 = (delta - d1) * (g2 - gamma) / denom;
    const double w22 = (delta - d1) * (gamma - g1) / denom;
    double radius = 0;
    radius += w11 * tab_radius[id1 * ng + ig1];
    radius += w12 * tab_radius[id1 * ng + ig2];
    radius += w21 * tab_radius[id2 * ng + ig1];
    radius += w22 * tab_radius[id2 * ng + ig2];
    const double Req = R / 2;
    const double a3 = radius * radius * radius;
    const double term1 = 4 * E0 * a3 / (3 * Req);
    const double term2 = 4 * std::sqrt(PI * a3 * gamma * E0);
    const V3 v = (term2 - term1) * d12n;
    out[0][0] = -v.x; out[0][1] = -v.y; out[0][2] = -v.z;
    out[1][0] = v.x; out[1][1] = v.y; out[1][2] = v.z;
    if (!constraint)
    {
        out[0][3] = -s * v.x; out[0][4] = -s * v.y; out[0][5] = -s * v.z;
        out[1][3] = t * v.x; out[1][4] = t * v.y; out[1][5] = t * v.z;
    }
    else
    {
        const V3 mv = v3(-v.x, -v.y, -v.z);
        const double w1 = dot(n1, mv), w2 = dot(n2, mv);
        const V3 a = (-w1) * n1 - v, b = w2 * n2 + v;
        out[0][3] = s * a.x; out[0][4] = s * a.y; out[0][5] = s * a.z;
        out[1][3] = t * b.x; out[1][4] = t * b.y; out[1][5] = t * b.z;
    }
}

// simulation.hpp:120-145 (calculateJKRContactRadii over an overlap mesh and a gamma mesh),
// overlap-major
inline std::vector<double> jkr_radius_table2(const std::vector<double>& overlaps,
                                             const std::vector<double>& gammas, double R, double E0)
{
    std::vector<double> radii(overlaps.size() * gammas.size());
    for (size_t i = 0; i < overlaps.size(); ++i)
        for (size_t j = 0; j < gammas.size(); ++j)
            radii[i * gammas.size() + j] = jkr_contact_radius(overlaps[i], R / 2, E0, gammas[j]);
    return radii;
}

// mechanics.hpp:1209-1350 (Hertz only) and :1390-1659 (Hertz + isotropic JKR), without
// the friction term (add_friction adds it).  Returns dE/dq (n x 6).  `constraint` selects
// include_constraint = true, the form velocity Verlet uses: the Hertz and hard-core rows
// become (s n) x v (mechanics.hpp:1298-1311, 1554-1566, 1608-1617).
// the pairs k0 <= k < k1 of the table, added into dEdq (n x 6) in table order
inline void cell_cell_forces_range(const Cells& cells, const Neighbors& nb, const Params3& p, bool constraint,
                                   int k0, int k1, Arr6& dEdq)
{
    const int n = cells.n;
    const double R = p.R, Rcell = p.Rcell;
    double pf[3]; repulsion_prefactors(p, pf);
    const bool adhesion = (p.adhesion_mode != 0);
    for (int k = k0; k < k1; ++k)
    {
        int i = nb.i[k], j = nb.j[k];
        V3 dij = v3(nb.dx[k], nb.dy[k], nb.dz[k]);
        double dist = norm(dij);
        double overlap = 2 * R - dist;
        if (!(overlap > 0)) continue;
        double si = nb.si[k], sj = nb.sj[k];
        V3 dijn = v3(dij.x / dist, dij.y / dist, dij.z / dist);
        double f[2][6];
        double max_overlap = 2 * (R - Rcell);
        double gamma = adhesion ? std::min(cells(i, C_GAMMA), cells(j, C_GAMMA)) : 0.0;
        if (adhesion && gamma > 0)
        {
            if (p.jkr_gammas.empty())
                jkr_forces(dij, R, p.E0, gamma, si, sj, p.jkr_overlaps, p.jkr_radii, max_overlap, f,
                           constraint, cell_n(cells, i), cell_n(cells, j));
            else
                jkr_forces_variable(dij, R, p.E0, gamma, si, sj, p.jkr_overlaps, p.jkr_gammas, p.jkr_radii2,
                                    max_overlap, f, constraint, cell_n(cells, i), cell_n(cells, j));
        }
        else
        {
            double magnitude;
            if (overlap <= max_overlap) magnitude = pf[0] * std::pow(overlap, 1.5);
            else
            {
                magnitude = pf[2];
                if (!adhesion) magnitude += pf[1] * std::pow(overlap - max_overlap, 1.5);
            }
            V3 vij = magnitude * dijn;
            f[0][0] = vij.x; f[0][1] = vij.y; f[0][2] = vij.z;
            f[1][0] = -vij.x; f[1][1] = -vij.y; f[1][2] = -vij.z;
            if (!constraint)
            {
                f[0][3] = si * vij.x; f[0][4] = si * vij.y; f[0][5] = si * vij.z;
                f[1][3] = -sj * vij.x; f[1][4] = -sj * vij.y; f[1][5] = -sj * vij.z;
            }
            else
            {
                const V3 ti = cross(si * cell_n(cells, i), vij);
                const V3 tj = cross(sj * cell_n(cells, j), v3(-vij.x, -vij.y, -vij.z));
                f[0][3] = ti.x; f[0][4] = ti.y; f[0][5] = ti.z;
                f[1][3] = tj.x; f[1][4] = tj.y; f[1][5] = tj.z;
            }
        }
        for (int c = 0; c < 6; ++c) { A6(dEdq, n, i, c) += f[0][c]; A6(dEdq, n, j, c) += f[1][c]; }
        if (adhesion && overlap > 2 * (R - Rcell))
        {
            double magnitude = pf[1] * std::pow(overlap - 2 * (R - Rcell), 1.5);
            V3 vij = magnitude * dijn;
            double h[2][6] = {{vij.x, vij.y, vij.z, si * vij.x, si * vij.y, si * vij.z},
                              {-vij.x, -vij.y, -vij.z, -sj * vij.x, -sj * vij.y, -sj * vij.z}};
            if (constraint)
            {
                const V3 ti = cross(si * cell_n(cells, i), vij);
                const V3 tj = cross(sj * cell_n(cells, j), v3(-vij.x, -vij.y, -vij.z));
                h[0][3] = ti.x; h[0][4] = ti.y; h[0][5] = ti.z;
                h[1][3] = tj.x; h[1][4] = tj.y; h[1][5] = tj.z;
            }
            for (int c = 0; c < 6; ++c) { A6(dEdq, n, i, c) += h[0][c]; A6(dEdq, n, j, c) += h[1][c]; }
        }
    }
}

// mechanics.hpp:1209-1350, 1390-1659 (cellCellInteractionForces): the pair loop in table
// order.  With cpu_optimized, each OpenMP thread sums a contiguous range of pairs into its
// own buffer and the buffers are added per cell in thread order (the sums then differ
// from the table-order ones by rounding only).
inline Arr6 cell_cell_forces(const Cells& cells, const Neighbors& nb, const Params3& p,
                             bool constraint = false)
{
    const int n = cells.n, m = nb.size();
    Arr6 dEdq((size_t)n * 6, 0.0);
    if (m == 0) return dEdq;
    if (!p.cpu_optimized)
    {
        cell_cell_forces_range(cells, nb, p, constraint, 0, m, dEdq);
        return dEdq;
    }
    const int T = std::max(1, std::min(omp_get_max_threads(), m));
    std::vector<Arr6> part((size_t)T);
    #pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const int k0 = (int)((long long)m * t / nt), k1 = (int)((long long)m * (t + 1) / nt);
        part[t].assign((size_t)n * 6, 0.0);
        cell_cell_forces_range(cells, nb, p, constraint, k0, k1, part[t]);
        #pragma omp barrier
        #pragma omp for
        for (int e = 0; e < n * 6; ++e)
        {
            double acc = 0.0;
            for (int u = 0; u < nt; ++u) acc += part[u][e];
            dEdq[e] = acc;
        }
    }
    return dEdq;
}

// mechanics.hpp:673-780 (cellSurfaceRepulsionForces).  With `constraint`
// (include_constraint) the nz row is replaced by x, y torques
// -2 E0 (ny, -nx) ((1 - nz^2) I2(1) + sqrt(R) nz^2 I2(1/2)) (mechanics.hpp:718-755).
inline Arr6 cell_surface_repulsion_forces(const Cells& cells, const std::vector<double>& ss,
                                          double R, double E0, const std::vector<int>& assume_2d,
                                          bool multithread, bool constraint = false)
{
    const int n = cells.n;
    Arr6 dEdq((size_t)n * 6, 0.0);
    const double prefactor0 = 2 * E0;
    const double prefactor1 = (8. / 3.) * E0 * std::pow(R, 0.5);
    const double prefactor2 = 2 * E0 * std::pow(R, 0.5);
    #pragma omp parallel for if(multithread)
    for (int i = 0; i < n; ++i)
    {
        double rz = cells(i, C_RZ), nz = cells(i, C_NZ), hl = cells(i, C_HALF_L);
        if (assume_2d[i])
        {
            double ph = R - rz;
            if (ph > 0) A6(dEdq, n, i, 2) = -prefactor0 * ph * cells(i, C_L);
        }
        else
        {
            double nz2 = nz * nz;
            double int1 = integral1(rz, nz, R, hl, 1.0, ss[i]);
            double int2 = integral1(rz, nz, R, hl, 0.5, ss[i]);
            A6(dEdq, n, i, 2) = -prefactor0 * ((1.0 - nz2) * int1 + std::sqrt(R) * nz2 * int2);
            if (constraint)
            {
                double i3 = integral2(rz, nz, R, hl, 1.0, ss[i]);
                double i4 = integral2(rz, nz, R, hl, 0.5, ss[i]);
                double cx = cells(i, C_NY), cy = -cells(i, C_NX);
                double w = (1.0 - nz2) * i3 + std::sqrt(R) * nz2 * i4;
                A6(dEdq, n, i, 3) = -prefactor0 * cx * w;
                A6(dEdq, n, i, 4) = -prefactor0 * cy * w;
                continue;
            }
            double int3 = integral1(rz, nz, R, hl, 2.0, ss[i]);
            double int4 = integral2(rz, nz, R, hl, 1.0, ss[i]);
            double int5 = integral1(rz, nz, R, hl, 1.5, ss[i]);
            double int6 = integral2(rz, nz, R, hl, 0.5, ss[i]);
            double& d5 = A6(dEdq, n, i, 5);
            d5 -= prefactor0 * nz * int3;
            d5 -= prefactor0 * (1 - nz2) * int4;
            d5 += prefactor1 * nz * int5;
            d5 -= prefactor2 * nz2 * int6;
        }
    }
    return dEdq;
}

// mechanics.hpp:800-910 (cellSurfaceAdhesionForces).  With `constraint`
// (include_constraint) the nz row is replaced by x, y torques (mechanics.hpp:845-886).
inline Arr6 cell_surface_adhesion_forces(const Cells& cells, const std::vector<double>& ss,
                                         double R, const std::vector<int>& assume_2d,
                                         bool multithread, bool constraint = false)
{
    const int n = cells.n;
    Arr6 dEdq((size_t)n * 6, 0.0);
    const double prefactor0 = std::pow(R, 0.5) / 2;
    const double prefactor1 = 2 * PI * R;
    const double prefactor2 = 2 * std::pow(R, 0.5);
    #pragma omp parallel for if(multithread)
    for (int i = 0; i < n; ++i)
    {
        double rz = cells(i, C_RZ), nz = cells(i, C_NZ), hl = cells(i, C_HALF_L);
        double sig = cells(i, C_SIGMA0);
        if (assume_2d[i])
        {
            double ph = R - rz;
            if (ph > 0) A6(dEdq, n, i, 2) = sig * prefactor0 * cells(i, C_L) / std::pow(ph, 0.5);
        }
        else
        {
            double nz2 = nz * nz;
            double int1 = integral1(rz, nz, R, hl, -0.5, ss[i]);
            double term2 = 0.0;
            if (std::fabs(ss[i]) < hl) term2 = (prefactor1 / 2) * nz;
            double d2 = prefactor0 * (1 - nz2) * int1 + term2;
            A6(dEdq, n, i, 2) = d2 * sig;
            if (constraint)
            {
                double i2 = integral2(rz, nz, R, hl, -0.5, ss[i]);
                double cx = cells(i, C_NY), cy = -cells(i, C_NX);
                double w1 = 0, w2 = 0;
                if (std::fabs(ss[i]) < hl)
                {
                    w1 = (prefactor1 / 2) * ss[i] * nz * cx;
                    w2 = (prefactor1 / 2) * ss[i] * nz * cy;
                }
                A6(dEdq, n, i, 3) = (prefactor0 * (1 - nz2) * i2 * cx - w1) * sig;
                A6(dEdq, n, i, 4) = (prefactor0 * (1 - nz2) * i2 * cy - w2) * sig;
                continue;
            }
            double int2 = integral1(rz, nz, R, hl, 0.5, ss[i]);
            double int3 = integral2(rz, nz, R, hl, -0.5, ss[i]);
            double int4 = integral4(nz, hl, ss[i]);
            double term4 = 0.0;
            if (std::fabs(ss[i]) < hl) term4 = (prefactor1 / 2) * (R - rz);
            double d5 = 0;
            d5 += prefactor2 * nz * int2;
            d5 += prefactor0 * (1 - nz2) * int3;
            d5 -= prefactor1 * nz * int4;
            d5 += term4;
            A6(dEdq, n, i, 5) = d5 * sig;
        }
    }
    return dEdq;
}

// mechanics.hpp:1031-1175 (cellCellFrictionForces, include_constraint = false), as
// cellCellInteractionForces adds it when friction_mode is KINETIC (mechanics.hpp:1339-1346,
// dz_threshold 1e-3).  At each overlapping pair the force on cell i is
// -eta sqrt(Req overlap) times the tangential part of the relative velocity of the two
// contact points (each cell's dr + s dn from its velocity columns), eta the smaller of the two
// cells' coefficients in column eta_col.  With coulomb_coeff > 0 its norm is capped at
// coulomb_coeff (4/3) E0 sqrt(Req) overlap^(3/2).  A contact whose distance vector is nearly
// horizontal (|dz / d| < dz_threshold) between two contact points below 1.01 R is taken in the
// xy-plane (surface present only).  Returns dE/dq (n x 6): minus the force and torque.
inline Arr6 cell_cell_friction_forces(const Cells& cells, const Neighbors& nb, double R, double E0,
                                      int eta_col, double coulomb_coeff, bool no_surface,
                                      double dz_threshold, bool constraint = false)
{
    const int n = cells.n, m = nb.size();
    Arr6 dEdq((size_t)n * 6, 0.0);
    if (m == 0) return dEdq;
    const double Req = R / 2;
    for (int k = 0; k < m; ++k)
    {
        const int i = nb.i[k], j = nb.j[k];
        V3 dij = v3(nb.dx[k], nb.dy[k], nb.dz[k]);
        const double dist = norm(dij);
        double overlap = 2 * R - dist;
        if (!(overlap > 0)) continue;
        const double si = nb.si[k], sj = nb.sj[k];
        V3 dijn = v3(dij.x / dist, dij.y / dist, dij.z / dist);
        const V3 ri = cell_r(cells, i), ni = cell_n(cells, i);
        const V3 rj = cell_r(cells, j), nj = cell_n(cells, j);
        const double eta = std::min(cells(i, eta_col), cells(j, eta_col));
        bool flat = false;
        if (!no_surface && std::fabs(dijn.z) < dz_threshold)
        {
            const V3 pi = ri + si * ni, pj = rj + sj * nj;
            flat = (pi.z < 1.01 * R && pj.z < 1.01 * R);
        }
        const V3 vi = v3(cells(i, C_DRX), cells(i, C_DRY), cells(i, C_DRZ)) +
                      si * v3(cells(i, C_DNX), cells(i, C_DNY), cells(i, C_DNZ));
        const V3 vj = v3(cells(j, C_DRX), cells(j, C_DRY), cells(j, C_DRZ)) +
                      sj * v3(cells(j, C_DNX), cells(j, C_DNY), cells(j, C_DNZ));
        V3 rv = vi - vj;
        if (flat)
        {
            dij.z = 0;
            const double d2 = norm(dij);
            dijn = v3(dij.x / d2, dij.y / d2, dij.z / d2);
            overlap = 2 * R - d2;
            rv.z = 0;
        }
        const V3 vt = rv - dot(rv, dijn) * dijn;
        V3 force = (-eta * std::sqrt(Req * overlap)) * vt;
        if (coulomb_coeff > 0)
        {
            const double fn = norm(force);
            const double max_norm = coulomb_coeff * (4. / 3.) * E0 * std::sqrt(Req) * std::pow(overlap, 1.5);
            if (fn > max_norm)
            {
                const double scale = max_norm / fn;
                force = v3(force.x * scale, force.y * scale, force.z * scale);
            }
        }
        // torques s force, or (s n) x force with include_constraint (mechanics.hpp:1152-1161)
        const V3 ti = constraint ? cross(si * ni, force) : si * force;
        const V3 tj = constraint ? cross(sj * nj, v3(-force.x, -force.y, -force.z)) : (-sj) * force;
        const double hi[6] = {-force.x, -force.y, -force.z, -ti.x, -ti.y, -ti.z};
        const double hj[6] = {force.x, force.y, force.z, -tj.x, -tj.y, -tj.z};
        for (int c = 0; c < 6; ++c) { A6(dEdq, n, i, c) += hi[c]; A6(dEdq, n, j, c) += hj[c]; }
    }
    return dEdq;
}

// cellCellInteractionForces' friction term (mechanics.hpp:1339-1346) added onto the pair
// forces: the friction coefficient column is 22 with adhesion on, 21 without
// (simulation.hpp:1184-1186).
inline void add_friction(Arr6& cc, const Cells& cells, const Neighbors& nb, const Params3& p,
                         bool constraint = false)
{
    if (p.friction_mode == 0) return;
    const int eta_col = p.adhesion_mode != 0 ? 22 : 21;
    if (cells.ncols <= eta_col) throw std::runtime_error("friction needs the cell-cell friction column");
    Arr6 fr = cell_cell_friction_forces(cells, nb, p.R, p.E0, eta_col, p.cell_cell_coulomb_coeff,
                                        p.no_surface != 0, 1e-3, constraint);
    for (size_t k = 0; k < cc.size(); ++k) cc[k] += fr[k];
}

// mechanics.hpp:1702-1769 (getConservativeForces): -(dE_cc) - dE_rep - dE_adh
inline Arr6 get_conservative_forces(const Cells& cells, const Neighbors& nb, const Params3& p,
                                    const std::vector<int>& assume_2d, bool multithread,
                                    const Arr6* dEdq_cc_cached = nullptr, bool constraint = false)
{
    const int n = cells.n;
    std::vector<double> ss(n);
    for (int i = 0; i < n; ++i)
        ss[i] = assume_2d[i] ? std::numeric_limits<double>::quiet_NaN()
                             : sstar(cells(i, C_RZ), cells(i, C_NZ), p.R);
    Arr6 cc = dEdq_cc_cached ? *dEdq_cc_cached : cell_cell_forces(cells, nb, p, constraint);
    add_friction(cc, cells, nb, p, constraint);   // velocity- and position-dependent: every stage
    Arr6 rep((size_t)n * 6, 0.0), adh((size_t)n * 6, 0.0);
    if (!p.no_surface)
    {
        rep = cell_surface_repulsion_forces(cells, ss, p.R, p.E0, assume_2d, multithread, constraint);
        adh = cell_surface_adhesion_forces(cells, ss, p.R, assume_2d, multithread, constraint);
    }
    Arr6 out((size_t)n * 6);
    for (size_t k = 0; k < out.size(); ++k) out[k] = ((-cc[k]) - rep[k]) - adh[k];
    return out;
}

// mechanics.hpp:1918-1959 (normalizeOrientations)
inline void normalize_orientations(Cells& cells)
{
    for (int i = 0; i < cells.n; ++i)
    {
        double nx = cells(i, C_NX), ny = cells(i, C_NY), nz = cells(i, C_NZ);
        double nrm = std::sqrt((nx * nx + ny * ny) + nz * nz);
        cells(i, C_NX) = nx / nrm; cells(i, C_NY) = ny / nrm; cells(i, C_NZ) = nz / nrm;
    }
    for (int i = 0; i < cells.n; ++i)
    {
        if (cells(i, C_NZ) < 0)
        {
            cells(i, C_NX) *= -1; cells(i, C_NY) *= -1; cells(i, C_NZ) *= -1;
        }
    }
}

// mechanics.hpp:2011-2347 (getVelocities); cell-cell friction enters through
// get_conservative_forces.  `noise` is n x 6.
inline Arr6 get_velocities(const Cells& cells, const Neighbors& nb, const Params3& p,
                           const std::vector<int>& assume_2d, const Arr6& noise,
                           bool multithread, const Arr6* dEdq_cc_cached = nullptr)
{
    const int n = cells.n;
    const double R = p.R, E0 = p.E0;
    const double coul = p.cell_surface_coulomb_coeff;
    Arr6 v((size_t)n * 6, 0.0);
    std::vector<double> ss(n);
    for (int i = 0; i < n; ++i)
        ss[i] = assume_2d[i] ? std::numeric_limits<double>::quiet_NaN()
                             : sstar(cells(i, C_RZ), cells(i, C_NZ), R);
    Arr6 F = get_conservative_forces(cells, nb, p, assume_2d, multithread, dEdq_cc_cached);
    for (size_t k = 0; k < F.size(); ++k) F[k] += noise[k];
    #pragma omp parallel for if(multithread)
    for (int i = 0; i < n; ++i)
    {
        const double rz = cells(i, C_RZ), nx = cells(i, C_NX), ny = cells(i, C_NY), nz = cells(i, C_NZ);
        const double l = cells(i, C_L), hl = cells(i, C_HALF_L);
        const double eta0 = cells(i, C_ETA0);
        double f[6]; for (int k = 0; k < 6; ++k) f[k] = A6c(F, n, i, k);
        double out[6] = {0, 0, 0, 0, 0, 0};
        bool contacting = false;
        if (!assume_2d[i])
        {
            double z1 = rz - hl * nz, z2 = rz + hl * nz;
            contacting = (z1 < R || z2 < R);
        }
        else contacting = (rz < R);
        if (p.no_surface || !contacting)
        {
            double K = eta0 * l;
            double L = K * l * l / 12;
            double mult = -((nx * f[3] + ny * f[4]) + nz * f[5]);
            out[0] = f[0] / K; out[1] = f[1] / K; out[2] = f[2] / K;
            out[3] = (f[3] + mult * nx) / L; out[4] = (f[4] + mult * ny) / L; out[5] = (f[5] + mult * nz) / L;
        }
        else if (assume_2d[i])
        {
            double K, L;
            if (coul == 0)
            {
                double a = std::sqrt(R * (R - rz));
                double eta_c = eta0 + cells(i, C_ETA1) * a / R;
                K = eta_c * l;
                L = K * l * l / 12;
            }
            else
            {
                double K_vis = eta0 * l;
                double L_vis = K_vis * l * l / 12;
                double a = std::sqrt(R * (R - rz));
                double K_fric = cells(i, C_ETA1) * l * a / R;
                double drx = cells(i, C_DRX), dry = cells(i, C_DRY);
                double drxy = std::sqrt(drx * drx + dry * dry);
                double friction_norm = K_fric * drxy;
                double max_norm = coul * (2 * E0 * (R - rz) * l);
                if (friction_norm > max_norm)
                {
                    double eta1_tr = max_norm * R / (drxy * l * a);
                    K_fric = eta1_tr * l * a / R;
                }
                double L_fric = K_fric * l * l / 12;
                K = K_vis + K_fric;
                L = L_vis + L_fric;
            }
            double mult = -(nx * f[3] + ny * f[4]);
            out[0] = f[0] / K; out[1] = f[1] / K;
            out[3] = (f[3] + mult * nx) / L; out[4] = (f[4] + mult * ny) / L;
            out[2] = f[2] / (eta0 * l);
            out[5] = 12 * f[5] / (eta0 * l * l * l);
        }
        else
        {
            double eta1 = cells(i, C_ETA1);
            double A1, A2, A3;
            area_integrals(rz, nz, R, hl, ss[i], A1, A2, A3);
            if (coul > 0)
            {
                double drx = cells(i, C_DRX), dry = cells(i, C_DRY);
                double dnx = cells(i, C_DNX), dny = cells(i, C_DNY);
                double drxy = std::sqrt(drx * drx + dry * dry);
                double dnxy = std::sqrt(dnx * dnx + dny * dny);
                double friction_norm = A1 * drxy;
                friction_norm += A2 * dnxy;
                friction_norm *= (eta1 / R);
                double max_norm = (1 - nz * nz) * integral1(rz, nz, R, hl, 1, ss[i]);
                max_norm += std::sqrt(R) * nz * nz * integral1(rz, nz, R, hl, 0.5, ss[i]);
                max_norm *= (2 * E0 * coul);
                if (friction_norm > max_norm)
                    eta1 = max_norm * R / (A1 * drxy + A2 * dnxy);
            }
            const double c1 = eta0 * l + (eta1 / R) * A1;
            const double c2 = eta0 * l;
            const double c3 = c2 * l * l / 12 + (eta1 / R) * A3;
            const double c4 = c2 * l * l / 12;
            const double c5 = (eta1 / R) * A2;
            const double term1 = c3 - (c5 * c5 / c1);
            const double w4 = f[3] - f[0] * (c5 / c1);
            const double w5 = f[4] - f[1] * (c5 / c1);
            const double nx2 = nx / term1, ny2 = ny / term1, nz2 = nz / c4;
            const double alpha = 2 * ((nx * nx2 + ny * ny2) + nz * nz2);
            const double beta = -((w4 * nx2 + w5 * ny2) + f[5] * nz2);
            const double lambda = beta / alpha;
            out[5] = (f[5] + 2 * nz * lambda) / c4;
            out[4] = (w5 + 2 * ny * lambda) / term1;
            out[3] = (w4 + 2 * nx * lambda) / term1;
            out[2] = f[2] / c2;
            out[1] = (f[1] - c5 * out[4]) / c1;
            out[0] = (f[0] - c5 * out[3]) / c1;
        }
        for (int k = 0; k < 6; ++k) A6(v, n, i, k) = out[k];
    }
    return v;
}

// Noise for one RK attempt (mechanics.hpp:2489-2510): uniform on
// [-max, max] per component, drawn once per stepRungeKuttaAdaptive call.
// Counter policy: (iter, attempt, cell, pair-of-components).
inline Arr6 sample_noise(int n, const Params3& p, int iter, int attempt)
{
    Arr6 noise((size_t)n * 6, 0.0);
    if (!(p.max_rxy_noise > 0 || p.max_rz_noise > 0 || p.max_nxy_noise > 0 || p.max_nz_noise > 0))
        return noise;
    const double mx[6] = {p.max_rxy_noise, p.max_rxy_noise, p.max_rz_noise,
                          p.max_nxy_noise, p.max_nxy_noise, p.max_nz_noise};
    if (p.stream)
    {
        for (int i = 0; i < n; ++i)
            for (int c = 0; c < 6; ++c)
            {
                const double u = p.stream->uniform01();
                A6(noise, n, i, c) = -mx[c] + 2 * mx[c] * u;
            }
        return noise;
    }
    uint32_t k0, k1;
    rng_key(p.rng_seed, RNG_PURPOSE_NOISE, k0, k1);
    for (int i = 0; i < n; ++i)
    {
        for (int c = 0; c < 3; ++c)
        {
            Philox4 x = philox4x32_10((uint32_t)iter, (uint32_t)attempt, (uint32_t)i, (uint32_t)c, k0, k1);
            double u0 = philox_u01(x.v[0], x.v[1]), u1 = philox_u01(x.v[2], x.v[3]);
            A6(noise, n, i, 2 * c) = -mx[2 * c] + 2 * mx[2 * c] * u0;
            A6(noise, n, i, 2 * c + 1) = -mx[2 * c + 1] + 2 * mx[2 * c + 1] * u1;
        }
    }
    return noise;
}

// mechanics.hpp:2406-2612 (stepRungeKuttaAdaptive).  Returns the new cell
// array; `errors` receives the n x 6 embedded error estimate.  Pair forces are
// taken from the neighbor table, which this function never refreshes, so they
// are the same in every stage (include_constraint = false); `cc_once` computes
// them once instead of per stage, which changes no arithmetic.
inline Cells step_rk_adaptive(const Tableau& tab, const Cells& cells, const Neighbors& nb,
                              double dt, const Params3& p, int iter, int attempt, Arr6& errors,
                              bool cc_once = false)
{
    const int n = cells.n;
    std::vector<int> assume_2d(n);
    for (int i = 0; i < n; ++i) assume_2d[i] = (cells(i, C_NZ) < p.nz_threshold);
    Arr6 noise = sample_noise(n, p, iter, attempt);
    const int s = tab.s;
    const bool multithread = (n >= p.n_start_multithread);
    Arr6 cc;
    const Arr6* ccp = nullptr;
    if (cc_once) { cc = cell_cell_forces(cells, nb, p); ccp = &cc; }
    std::vector<Arr6> vel;
    vel.push_back(get_velocities(cells, nb, p, assume_2d, noise, multithread, ccp));
    for (int i = 1; i < s; ++i)
    {
        Arr6 mult((size_t)n * 6, 0.0);
        for (int j = 0; j < i; ++j)
            for (size_t k = 0; k < mult.size(); ++k) mult[k] += vel[j][k] * tab.a(i, j);
        Cells ci(cells);
        for (int c = 0; c < 6; ++c)
            for (int r = 0; r < n; ++r) ci(r, C_RX + c) += A6(mult, n, r, c) * dt;
        normalize_orientations(ci);
        vel.push_back(get_velocities(ci, nb, p, assume_2d, noise, multithread, ccp));
    }
    Cells cn(cells);
    Arr6 vf1((size_t)n * 6, 0.0), vf2((size_t)n * 6, 0.0);
    for (int i = 0; i < s; ++i)
        for (size_t k = 0; k < vf1.size(); ++k) { vf1[k] += vel[i][k] * tab.b[i]; vf2[k] += vel[i][k] * tab.bs[i]; }
    errors.assign((size_t)n * 6, 0.0);
    for (int c = 0; c < 6; ++c)
        for (int r = 0; r < n; ++r)
        {
            double d1 = A6(vf1, n, r, c) * dt, d2 = A6(vf2, n, r, c) * dt;
            cn(r, C_RX + c) += d1;
            A6(errors, n, r, c) = d1 - d2;
        }
    for (int c = 0; c < 6; ++c)
        for (int r = 0; r < n; ++r) cn(r, C_DRX + c) = A6(vf1, n, r, c);
    normalize_orientations(cn);
    return cn;
}

// simulation.hpp:1697-1705: max over cells/components of err / (tol (1 + |y0|)),
// floored at min_error (signed errors, as in the reference)
inline double max_scaled_error(const Cells& cells, const Arr6& errors, double tol, double min_error)
{
    const int n = cells.n;
    double mx = -std::numeric_limits<double>::infinity();
    for (int c = 0; c < 6; ++c)
        for (int r = 0; r < n; ++r)
        {
            double z = 1.0 + std::fabs(cells(r, C_RX + c));
            double v = A6c(errors, n, r, c) / (tol * z);
            if (v > mx) mx = v;
        }
    return std::max(mx, min_error);
}

// growth.hpp:51-57 (growCells)
inline void grow_cells(Cells& cells, double dt, double R)
{
    for (int i = 0; i < cells.n; ++i)
    {
        cells(i, C_L) += cells(i, C_GROWTH) * (4 * R / 3 + cells(i, C_L)) * dt;
        cells(i, C_HALF_L) = cells(i, C_L) / 2;
    }
}

// growth.hpp:82-117 (minDistToCell)
inline double min_dist_to_cell(const Cells& cells, int i)
{
    double mindist = std::numeric_limits<double>::infinity();
    for (int j = 0; j < cells.n; ++j)
    {
        if (i == j) continue;
        double d = norm(dist_cells(cells, i, j).d);
        if (d < mindist) mindist = d;
    }
    return mindist;
}

// utils.hpp:648-655 (standardNormal, Box-Muller) on two policy uniforms, with
// the deterministic log / cos of detmath.hpp
inline double standard_normal(double u, double v)
{
    double c = std::sqrt(-2 * det_log(u));
    double sn, cs;
    det_sincos(TWO_PI * v, sn, cs);
    return c * cs;
}

// utils.hpp:791-801 (rotateXY)
inline V3 rotate_xy(V3 n, double theta)
{
    double st, ct;
    det_sincos(theta, st, ct);
    return v3(ct * n.x + (-st) * n.y + 0 * n.z, st * n.x + ct * n.y + 0 * n.z, (0 * n.x + 0 * n.y) + 1 * n.z);
}

// utils.hpp:814-829 (rotateOutOfXY)
inline V3 rotate_out_of_xy(V3 n, double theta)
{
    V3 v = v3(n.y * 1 - n.z * 0, n.z * 0 - n.x * 1, n.x * 0 - n.y * 0);   // n x z
    double nv = norm(v);
    v = v3(v.x / nv, v.y / nv, v.z / nv);
    double st, ct;
    det_sincos(theta, st, ct);
    V3 w = v3(v.y * n.z - v.z * n.y, v.z * n.x - v.x * n.z, v.x * n.y - v.y * n.x);   // v x n
    return v3(n.x * ct + w.x * st, n.y * ct + w.y * st, n.z * ct + w.z * st);
}

// Draw slots of one division try (policy): 0-3 angles, 4-5 length fraction,
// 6-7 mother growth rate, 8-9 daughter growth rate.
// growth-rate distribution of a cell's group: one distribution without switching, the
// group's own with it (growth.hpp:634-644 samples growth_dists[group - 1])
inline double growth_mean_of(const Params3& p, double group)
{
    return p.switch_mode == 0 ? p.growth_mean : p.group_growth_mean[(int)group == 1 ? 0 : 1];
}
inline double growth_std_of(const Params3& p, double group)
{
    return p.switch_mode == 0 ? p.growth_std : p.group_growth_std[(int)group == 1 ? 0 : 1];
}

inline double div_uniform(const Params3& p, int iter, int k, int tr, int slot)
{
    if (p.stream) return p.stream->uniform01();
    return rng_uniform(p.rng_seed, RNG_PURPOSE_DIVIDE, (uint32_t)iter, (uint32_t)k,
                       (uint32_t)tr, (uint32_t)slot);
}

// growth.hpp:166-426 (divideCells, one group).  Mothers keep their row
// (daughter 1); daughter 2 rows are appended in ascending mother order; IDs are
// max_id + 2k + 1 and max_id + 2k + 2.  `ntries_out` is the number of tries.
inline Cells divide_cells(const Cells& cells, std::vector<int>& parents, double t, const Params3& p,
                          const std::vector<int>& to_divide, int iter, int* ntries_out = nullptr)
{
    int n_divide = 0;
    for (int v : to_divide) n_divide += v;
    if (ntries_out) *ntries_out = 0;
    if (n_divide == 0) return cells;
    const int n = cells.n;
    const double R = p.R;
    std::vector<int> idx_divide;
    for (int i = 0; i < n; ++i) if (to_divide[i]) idx_divide.push_back(i);
    Cells total(n + n_divide, cells.ncols);
    std::vector<int> check_distance(n_divide, 1);
    const double mindist_default = 2 * p.Rcell;
    for (int m = 0; m < n_divide; ++m)
        if (min_dist_to_cell(cells, idx_divide[m]) < mindist_default) check_distance[m] = 0;
    std::vector<int> satisfies(n_divide, 0);
    for (int m = 0; m < n_divide; ++m) if (check_distance[m] == 0) satisfies[m] = 1;
    int ntries = 0;
    const int ntries_total = 10;
    auto sum = [](const std::vector<int>& v) { int s = 0; for (int x : v) s += x; return s; };
    while (ntries == 0 || (ntries < ntries_total && sum(satisfies) < n_divide))
    {
        for (int c = 0; c < cells.ncols; ++c)
            for (int r = 0; r < n; ++r) total(r, c) = cells(r, c);
        Cells nc(n_divide, cells.ncols);
        for (int m = 0; m < n_divide; ++m)
            for (int c = 0; c < cells.ncols; ++c) nc(m, c) = cells(idx_divide[m], c);
        std::vector<double> txy1(n_divide, 0), tz1(n_divide, 0), txy2(n_divide, 0), tz2(n_divide, 0);
        for (int m = 0; m < n_divide; ++m)
        {
            if (ntries < ntries_total - 1 && check_distance[m] == 1)
            {
                double bxy = p.daughter_angle_xy_bound, bz = p.daughter_angle_z_bound;
                txy1[m] = -bxy + 2 * bxy * div_uniform(p, iter, m, ntries, 0);
                if (!p.planar_division) tz1[m] = -bz + 2 * bz * div_uniform(p, iter, m, ntries, 1);
                txy2[m] = -bxy + 2 * bxy * div_uniform(p, iter, m, ntries, 2);
                if (!p.planar_division) tz2[m] = -bz + 2 * bz * div_uniform(p, iter, m, ntries, 3);
            }
        }
        for (int m = 0; m < n_divide; ++m)
        {
            V3 u = cell_n(nc, m);
            V3 a1 = rotate_out_of_xy(rotate_xy(u, txy1[m]), tz1[m]);
            V3 a2 = rotate_out_of_xy(rotate_xy(u, txy2[m]), tz2[m]);
            int im = idx_divide[m];
            total(im, C_NX) = a1.x; total(im, C_NY) = a1.y; total(im, C_NZ) = a1.z;
            nc(m, C_NX) = a2.x; nc(m, C_NY) = a2.y; nc(m, C_NZ) = a2.z;
        }
        for (int m = 0; m < n_divide; ++m)
        {
            // u before v, as standardNormal draws them (utils.hpp:648-655)
            const double u = div_uniform(p, iter, m, ntries, 4), v = div_uniform(p, iter, m, ntries, 5);
            double r = 0.5 + p.daughter_length_std * standard_normal(u, v);
            double M = (r < 0) ? 0.0 : (r > 1 ? 1.0 : r);
            int im = idx_divide[m];
            double Ld = total(im, C_L) - 2 * R;
            double L1 = M * Ld, L2 = (1 - M) * Ld;
            double div = -total(im, C_HALF_L) + L1 + R;
            double delta1 = L1 / 2 + R, delta2 = L2 / 2 + R;
            total(im, C_L) = L1; total(im, C_HALF_L) = L1 / 2;
            nc(m, C_L) = L2; nc(m, C_HALF_L) = L2 / 2;
            for (int c = 0; c < 3; ++c)
            {
                total(im, C_RX + c) = total(im, C_RX + c) + (div - delta1) * total(im, C_NX + c);
                nc(m, C_RX + c) = nc(m, C_RX + c) + (div + delta2) * nc(m, C_NX + c);
            }
            total(im, C_T0) = t; nc(m, C_T0) = t;
        }
        for (int m = 0; m < n_divide; ++m)
        {
            const double u = div_uniform(p, iter, m, ntries, 6), v = div_uniform(p, iter, m, ntries, 7);
            total(idx_divide[m], C_GROWTH) = growth_mean_of(p, total(idx_divide[m], C_GROUP)) +
                growth_std_of(p, total(idx_divide[m], C_GROUP)) * standard_normal(u, v);
        }
        for (int m = 0; m < n_divide; ++m)
        {
            const double u = div_uniform(p, iter, m, ntries, 8), v = div_uniform(p, iter, m, ntries, 9);
            nc(m, C_GROWTH) = growth_mean_of(p, nc(m, C_GROUP)) + growth_std_of(p, nc(m, C_GROUP)) *
                standard_normal(u, v);
        }
        for (int m = 0; m < n_divide; ++m)
            for (int c = 0; c < cells.ncols; ++c) total(n + m, c) = nc(m, c);
        std::vector<double> md1(n_divide, 0), md2(n_divide, 0);
        for (int m = 0; m < n_divide; ++m)
            if (check_distance[m] == 1) md1[m] = min_dist_to_cell(total, idx_divide[m]);
        for (int m = 0; m < n_divide; ++m)
            if (check_distance[m] == 1) md2[m] = min_dist_to_cell(total, n + m);
        for (int m = 0; m < n_divide; ++m)
            if (check_distance[m] == 1 && md1[m] >= mindist_default && md2[m] >= mindist_default)
                satisfies[m] = 1;
        ntries++;
    }
    if (ntries_out) *ntries_out = ntries;
    int max_id = (int)parents.size() - 1;
    for (int m = 0; m < n_divide; ++m)
    {
        int id1 = max_id + (2 * m + 1), id2 = max_id + (2 * m + 2);
        int parent_id = (int)total(idx_divide[m], C_ID);
        total(idx_divide[m], C_ID) = id1;
        total(n + m, C_ID) = id2;
        parents.push_back(parent_id);
        parents.push_back(parent_id);
    }
    return total;
}

// ------------------------------------------------------------------------
// Simulation loop body (simulation.hpp:1617-1864, switching, writing,
// basal_only and pole tracking excluded)
// ------------------------------------------------------------------------
// ------------------------------------------------------------------------
// Velocity Verlet (IntegrationMode::VELOCITY_VERLET = 0, simulation.hpp:1786-1798)
// ------------------------------------------------------------------------

// integrals.hpp:203-229 (integral3)
inline double integral3(double rz, double nz, double R, double half_l, double gamma, double ss)
{
    double term1 = 2 * integral2(rz, nz, R, half_l, gamma + 1, ss);
    double term2 = 0;
    if (ss > half_l)
    {
        double o1 = pow_e(phi(rz, nz, R, -half_l), gamma + 1);
        double o2 = pow_e(phi(rz, nz, R, half_l), gamma + 1);
        term2 = half_l * half_l * (o1 - o2);
    }
    else if (ss > -half_l)
    {
        term2 = half_l * half_l * pow_e(phi(rz, nz, R, -half_l), gamma + 1);
    }
    return (term1 + term2) / (nz * (gamma + 1));
}

// integrals.hpp:334-383 (areaIntegral1, areaIntegral2, areaIntegral3), each on its own as
// cellSurfaceFrictionForces calls them
inline double area_integral(int k, double rz, double nz, double R, double half_l, double ss)
{
    const double t = std::sqrt(R) * (1 - nz * nz);
    if (k == 1) return t * integral1(rz, nz, R, half_l, 0.5, ss) + PI * R * nz * nz * integral4(nz, half_l, ss);
    if (k == 2) return t * integral2(rz, nz, R, half_l, 0.5, ss) + PI * R * nz * nz * integral5(nz, half_l, ss);
    return t * integral3(rz, nz, R, half_l, 0.5, ss) + PI * R * nz * nz * integral6(nz, half_l, ss);
}

// mechanics.hpp:1784-1820 (ambientViscosityForces): eta0 l^3 dr and eta0 l^9 (n x dn) / 12,
// with the cube of the length as the reference computes it (li = pow(l, 3)).
inline Arr6 ambient_viscosity_forces(const Cells& cells)
{
    const int n = cells.n;
    Arr6 dEdq((size_t)n * 6, 0.0);
    for (int i = 0; i < n; ++i)
    {
        const V3 w = cross(cell_n(cells, i), v3(cells(i, C_DNX), cells(i, C_DNY), cells(i, C_DNZ)));
        const double eta = cells(i, C_ETA0), li = std::pow(cells(i, C_L), 3);
        const double a = eta * li, b = eta * li * li * li;
        A6(dEdq, n, i, 0) = a * cells(i, C_DRX); A6(dEdq, n, i, 1) = a * cells(i, C_DRY);
        A6(dEdq, n, i, 2) = a * cells(i, C_DRZ);
        A6(dEdq, n, i, 3) = b * w.x / 12; A6(dEdq, n, i, 4) = b * w.y / 12; A6(dEdq, n, i, 5) = b * w.z / 12;
    }
    return dEdq;
}

// mechanics.hpp:1821-1917 (cellSurfaceFrictionForces): friction eta1 / R times the contact
// area moments against the in-plane velocity q = (drx, dry, 0) and m, the in-plane part of
// (n x dn) x n; a horizontal cell uses its flat contact area sqrt(R (R - rz)) l.
inline Arr6 cell_surface_friction_forces(const Cells& cells, const std::vector<double>& ss, double R,
                                         const std::vector<int>& assume_2d)
{
    const int n = cells.n;
    Arr6 dEdq((size_t)n * 6, 0.0);
    for (int i = 0; i < n; ++i)
    {
        const V3 ni = cell_n(cells, i);
        const V3 w = cross(ni, v3(cells(i, C_DNX), cells(i, C_DNY), cells(i, C_DNZ)));
        const V3 q = v3(cells(i, C_DRX), cells(i, C_DRY), 0);
        const V3 m = v3(w.y * ni.z - w.z * ni.y, w.z * ni.x - w.x * ni.z, 0);
        const double eta = cells(i, C_ETA1);
        if (assume_2d[i])
        {
            const double ph = R - cells(i, C_RZ);
            if (ph > 0)
            {
                const double area = std::sqrt(R) * std::sqrt(ph) * cells(i, C_L);
                A6(dEdq, n, i, 0) = eta * q.x * area / R;
                A6(dEdq, n, i, 1) = eta * q.y * area / R;
                const double cz = ni.x * m.y - ni.y * m.x;
                const double l2 = cells(i, C_L) * cells(i, C_L);
                A6(dEdq, n, i, 5) = eta * cz * area * l2 / (12 * R);
            }
        }
        else
        {
            const double rz = cells(i, C_RZ), hl = cells(i, C_HALF_L);
            const double i1 = area_integral(1, rz, ni.z, R, hl, ss[i]);
            const double i2 = area_integral(2, rz, ni.z, R, hl, ss[i]);
            const double i3 = area_integral(3, rz, ni.z, R, hl, ss[i]);
            A6(dEdq, n, i, 0) = eta * (q.x * i1 + m.x * i2) / R;
            A6(dEdq, n, i, 1) = eta * (q.y * i1 + m.y * i2) / R;
            const V3 c1 = cross(ni, q), c2 = cross(ni, m);
            A6(dEdq, n, i, 3) = eta * (c1.x * i2 + c2.x * i3) / R;
            A6(dEdq, n, i, 4) = eta * (c1.y * i2 + c2.y * i3) / R;
            A6(dEdq, n, i, 5) = eta * (c1.z * i2 + c2.z * i3) / R;
        }
    }
    return dEdq;
}

// the forces of one half of a velocity-Verlet step (mechanics.hpp:2834-2862 and :2919-2947):
// the conservative forces in their include_constraint form plus the noise, minus the ambient
// viscosity, minus the cell-surface friction (capped row by row at
// cell_surface_coulomb_coeff times the constrained surface repulsion when that is positive)
inline Arr6 verlet_forces(const Cells& cells, const Neighbors& nb, const Params3& p, const Arr6& noise)
{
    const int n = cells.n;
    std::vector<int> a2(n);
    std::vector<double> ss(n);
    for (int i = 0; i < n; ++i)
    {
        a2[i] = cells(i, C_NZ) < p.nz_threshold;
        ss[i] = a2[i] ? std::numeric_limits<double>::quiet_NaN() : sstar(cells(i, C_RZ), cells(i, C_NZ), p.R);
    }
    Arr6 f = get_conservative_forces(cells, nb, p, a2, false, nullptr, true);
    for (size_t k = 0; k < f.size(); ++k) f[k] += noise[k];
    Arr6 amb = ambient_viscosity_forces(cells);
    for (size_t k = 0; k < f.size(); ++k) f[k] -= amb[k];
    if (!p.no_surface)
    {
        Arr6 csf = cell_surface_friction_forces(cells, ss, p.R, a2);
        if (p.cell_surface_coulomb_coeff > 0)
        {
            Arr6 rep = cell_surface_repulsion_forces(cells, ss, p.R, p.E0, a2, false, true);
            for (int i = 0; i < n; ++i)
            {
                // row norms of the six generalized components, summed in order (Eigen's
                // vectorised reduction may pair them otherwise: an ulp, only ever deciding a tie)
                double sf = 0, sr = 0;
                for (int c = 0; c < 6; ++c)
                {
                    sf += A6c(csf, n, i, c) * A6c(csf, n, i, c);
                    sr += A6c(rep, n, i, c) * A6c(rep, n, i, c);
                }
                const double fn = std::sqrt(sf), max_norm = p.cell_surface_coulomb_coeff * std::sqrt(sr);
                if (fn > max_norm)
                    for (int c = 0; c < 6; ++c) A6(csf, n, i, c) *= (max_norm / fn);
            }
        }
        for (size_t k = 0; k < f.size(); ++k) f[k] -= csf[k];
    }
    return f;
}

// the accelerations of one half step: forces / mass, and torques split along n and across it
// over the two moments of inertia (mechanics.hpp:2863-2877)
inline void verlet_accelerations(const Cells& cells, const Arr6& f, const std::vector<double>& mass,
                                 const std::vector<double>& mom_par, const std::vector<double>& mom_perp,
                                 std::vector<V3>& lin, std::vector<V3>& ang)
{
    const int n = cells.n;
    lin.resize(n); ang.resize(n);
    for (int i = 0; i < n; ++i)
    {
        const V3 ni = cell_n(cells, i);
        const V3 tq = v3(A6c(f, n, i, 3), A6c(f, n, i, 4), A6c(f, n, i, 5));
        const V3 tpar = dot(tq, ni) * ni, tperp = tq - tpar;
        lin[i] = v3(A6c(f, n, i, 0) / mass[i], A6c(f, n, i, 1) / mass[i], A6c(f, n, i, 2) / mass[i]);
        ang[i] = v3(tpar.x / mom_par[i], tpar.y / mom_par[i], tpar.z / mom_par[i]) +
                 v3(tperp.x / mom_perp[i], tperp.y / mom_perp[i], tperp.z / mom_perp[i]);
    }
}

// mechanics.hpp:2668-2996 (stepVelocityVerlet): half kick, drift of the two cell ends with the
// half-step velocity and angular velocity, refreshed neighbor distances, forces at the new
// state, second half kick; dn = omega x n.  rho is the cell density, M0 / volume of a cell of
// length L0 (simulation.hpp:1279-1290).
inline Cells step_velocity_verlet(const Cells& cells, const Neighbors& nb, double dt, const Params3& p,
                                  double rho, int iter)
{
    const int n = cells.n;
    const double R = p.R;
    Arr6 noise = sample_noise(n, p, iter, 0);
    std::vector<double> mass(n), mom_par(n), mom_perp(n);
    for (int i = 0; i < n; ++i)
    {
        const double length = cells(i, C_L);
        const double volume = PI * ((4. / 3.) * std::pow(R, 3) + R * R * length);
        mass[i] = rho * volume;
        const double diam = 2 * R, d2 = diam * diam, d3 = d2 * diam, d4 = d3 * diam;
        const double l2 = length * length, l3 = l2 * length;
        mom_par[i] = d4 * (length / 32 + diam / 60) * (rho * PI);
        mom_perp[i] = d2 * (4 * d3 + 15 * length * d2 + 20 * l2 * diam + 10 * l3) / 480 * (rho * PI);
    }
    std::vector<V3> omega(n);
    for (int i = 0; i < n; ++i)
        omega[i] = cross(cell_n(cells, i), v3(cells(i, C_DNX), cells(i, C_DNY), cells(i, C_DNZ)));
    Cells cn = cells;
    std::vector<V3> lin, ang;
    verlet_accelerations(cells, verlet_forces(cells, nb, p, noise), mass, mom_par, mom_perp, lin, ang);
    const double h = 0.5 * dt;
    std::vector<V3> w_half(n);
    for (int i = 0; i < n; ++i)
    {
        const V3 ri = cell_r(cells, i), ni = cell_n(cells, i);
        const double hl = cells(i, C_HALF_L);
        const V3 vi = v3(cells(i, C_DRX), cells(i, C_DRY), cells(i, C_DRZ)) + h * lin[i];
        const V3 wi = omega[i] + h * ang[i];
        w_half[i] = wi;
        const V3 pi = ri - hl * ni, qi = ri + hl * ni;
        const V3 c = cross(wi, pi - qi);
        const V3 half = v3(c.x / 2, c.y / 2, c.z / 2);
        const V3 pn = pi + dt * (vi + half), qn = qi + dt * (vi - half);
        const V3 rn = v3((pn.x + qn.x) / 2, (pn.y + qn.y) / 2, (pn.z + qn.z) / 2);
        const double length = cells(i, C_L);
        const V3 nn = v3((qn.x - pn.x) / length, (qn.y - pn.y) / length, (qn.z - pn.z) / length);
        const V3 dni = cross(wi, ni);
        cn(i, C_RX) = rn.x; cn(i, C_RY) = rn.y; cn(i, C_RZ) = rn.z;
        cn(i, C_NX) = nn.x; cn(i, C_NY) = nn.y; cn(i, C_NZ) = nn.z;
        cn(i, C_DRX) = vi.x; cn(i, C_DRY) = vi.y; cn(i, C_DRZ) = vi.z;
        cn(i, C_DNX) = dni.x; cn(i, C_DNY) = dni.y; cn(i, C_DNZ) = dni.z;
    }
    normalize_orientations(cn);
    Neighbors nb2 = nb;
    update_neighbor_distances(cn, nb2);
    verlet_accelerations(cn, verlet_forces(cn, nb2, p, noise), mass, mom_par, mom_perp, lin, ang);
    for (int i = 0; i < n; ++i)
    {
        cn(i, C_DRX) += h * lin[i].x; cn(i, C_DRY) += h * lin[i].y; cn(i, C_DRZ) += h * lin[i].z;
        const V3 wf = w_half[i] + h * ang[i];
        const V3 dni = cross(wf, cell_n(cn, i));
        cn(i, C_DNX) = dni.x; cn(i, C_DNY) = dni.y; cn(i, C_DNZ) = dni.z;
    }
    normalize_orientations(cn);
    return cn;
}

// ------------------------------------------------------------------------
// Phenotype switching, attribute / gamma ramps, local viscosity, basal-only
// compaction (the f4 row).  Random draws follow the Philox policy, purpose SWITCH,
// counters (iteration, cell or pair, slot).
// ------------------------------------------------------------------------
inline double switch_uniform(const Params3& p, int iter, int k, int slot)
{
    if (p.stream) return p.stream->uniform01();
    return rng_uniform(p.rng_seed, RNG_PURPOSE_SWITCH, (uint32_t)iter, (uint32_t)k, (uint32_t)slot, 0u);
}

inline double switch_growth(const Params3& p, int group0, int iter, int k, int slot)
{
    const double u = switch_uniform(p, iter, k, slot), v = switch_uniform(p, iter, k, slot + 1);
    return p.group_growth_mean[group0] + p.group_growth_std[group0] * standard_normal(u, v);
}

// switch.hpp:45-95 (switchGroupsMarkov): each cell leaves its group g for group j when a
// uniform r falls in [sum of the earlier probabilities, + dt rate(g, j)), and then draws a
// growth rate from group j's distribution.
inline int switch_groups_markov(Cells& cells, const Params3& p, double dt, int iter)
{
    int switched = 0;
    for (int i = 0; i < cells.n; ++i)
    {
        const int group = (int)cells(i, C_GROUP) - 1;
        const double r = switch_uniform(p, iter, i, 0);
        double total = 0;
        for (int j = 0; j < 2; ++j)
        {
            if (j == group) continue;
            const double prob = dt * p.switch_rates[group * 2 + j];
            if (r > total && r < total + prob)
            {
                cells(i, C_GROUP) = j + 1;
                cells(i, C_GROWTH) = switch_growth(p, j, iter, i, 2);
                ++switched;
                break;
            }
            total += prob;
        }
    }
    return switched;
}

// switch.hpp:97-142 (switchGroupsInherit): for each pair of daughters of group g, with
// probability 1 - P(g, g) one of the two, chosen by a second uniform, moves to the other
// group and draws that group's growth rate.
inline int switch_groups_inherit(Cells& cells, const std::vector<std::pair<int, int> >& pairs,
                                 const Params3& p, int iter)
{
    int switched = 0;
    for (size_t q = 0; q < pairs.size(); ++q)
    {
        const int i = pairs[q].first, j = pairs[q].second;
        const int group = (int)cells(i, C_GROUP) - 1;
        const double r = switch_uniform(p, iter, (int)q, 4);
        double total = p.switch_rates[group * 2 + group];
        if (!(r > total)) continue;
        for (int k = 0; k < 2; ++k)
        {
            if (k == group) continue;
            const double prob = p.switch_rates[group * 2 + k];
            if (r > total && r < total + prob)
            {
                const int which = switch_uniform(p, iter, (int)q, 5) < 0.5 ? i : j;
                cells(which, C_GROUP) = k + 1;
                cells(which, C_GROWTH) = switch_growth(p, k, iter, (int)q, 6);
                ++switched;
                break;
            }
            total += prob;
        }
    }
    return switched;
}

// simulation.hpp:1872-1938: each switched attribute moves toward its group's target at
// |target1 - target2| / switch_timescale per unit time (at once with a zero timescale),
// stopping at the target.
inline void ramp_attributes(Cells& cells, const Params3& p, double dt)
{
    for (int k = 0; k < p.n_attributes; ++k)
    {
        const int col = p.attr_col[k];
        const double t1 = p.attr_target[0][k], t2 = p.attr_target[1][k];
        const double rate = p.switch_timescale == 0 ? std::numeric_limits<double>::infinity()
                                                    : std::fabs(t1 - t2) / p.switch_timescale;
        for (int i = 0; i < cells.n; ++i)
        {
            const bool g1 = (int)cells(i, C_GROUP) == 1;
            const double own = g1 ? t1 : t2, other = g1 ? t2 : t1;
            double& v = cells(i, col);
            if (p.switch_timescale == 0 && v != own) v = own;
            else if (own > other && v < own) { v += rate * dt; if (v > own) v = own; }
            else if (own < other && v > own) { v -= rate * dt; if (v < own) v = own; }
            else if (t1 == t2 && v != own) v = own;
        }
    }
}

// simulation.hpp:1940-1957: gamma rises toward max_gamma in group 1 and falls toward 0 in
// group 2 at max_gamma / switch_timescale (at once with a zero timescale; simulation.hpp:1361-1364).
inline void ramp_gamma(Cells& cells, const Params3& p, double dt)
{
    const double rate = p.switch_timescale == 0 ? std::numeric_limits<double>::infinity()
                                                : p.max_gamma / p.switch_timescale;
    for (int i = 0; i < cells.n; ++i)
    {
        double& g = cells(i, C_GAMMA);
        if ((int)cells(i, C_GROUP) == 1)
        {
            if (g < p.max_gamma) { g += rate * dt; if (g > p.max_gamma) g = p.max_gamma; }
        }
        else if (g > 0) { g -= rate * dt; if (g < 0) g = 0; }
    }
}

// simulation.hpp:1958-2020: the ambient viscosity of each cell interpolates between its
// group's limits by the share of group-1 cells among its contacts (distance < 2R), the
// denominator at least max_coordination_number, saturating at that many group-1 contacts.
inline void modulate_viscosity(Cells& cells, const Neighbors& nb, const Params3& p)
{
    const int n = cells.n;
    std::vector<int> total(n, 0), g1(n, 0);
    for (int k = 0; k < nb.size(); ++k)
    {
        const int i = nb.i[k], j = nb.j[k];
        if (norm(v3(nb.dx[k], nb.dy[k], nb.dz[k])) < 2 * p.R)
        {
            total[i] += 1; total[j] += 1;
            if ((int)cells(i, C_GROUP) == 1) g1[j] += 1;
            if ((int)cells(j, C_GROUP) == 1) g1[i] += 1;
        }
    }
    for (int i = 0; i < n; ++i)
    {
        const int group = (int)cells(i, C_GROUP) - 1;
        const double vmin = p.viscosity_lims[group * 2], vmax = p.viscosity_lims[group * 2 + 1];
        if (g1[i] >= p.max_coordination_number) cells(i, C_ETA0) = vmax;
        else
        {
            const double ratio = (double)g1[i] / (double)std::max(total[i], p.max_coordination_number);
            cells(i, C_ETA0) = vmin + ratio * (vmax - vmin);
        }
    }
}

// simulation.hpp:1831-1856: with the surface present, keep only the cells whose deepest
// overlap R - rz + half_l nz exceeds basal_min_overlap; returns how many were dropped.
inline int basal_compact(Cells& cells, const Params3& p)
{
    std::vector<int> keep;
    for (int i = 0; i < cells.n; ++i)
        if (p.R - cells(i, C_RZ) + cells(i, C_HALF_L) * cells(i, C_NZ) > p.basal_min_overlap) keep.push_back(i);
    const int dropped = cells.n - (int)keep.size();
    if (dropped == 0) return 0;
    Cells kept((int)keep.size(), cells.ncols);
    for (int c = 0; c < cells.ncols; ++c)
        for (size_t r = 0; r < keep.size(); ++r) kept((int)r, c) = cells(keep[r], c);
    cells = kept;
    return dropped;
}

struct LoopState {
    Cells cells;
    Neighbors nb;
    std::vector<int> parents;
    double t = 0, dt = 0;
    int iter = 0;
    // statistics
    long long attempts = 0, rebuilds = 0, divisions = 0;
    double last_max_error = 0;
    double prev_accepted_error = 0;   // E of the step before the last accepted one (0: none yet)
    long long rejected = 0;           // iterations whose first attempt failed the error test
};

// The PI proposal after an accepted step of dt with scaled error E, E_prev the error of
// the accepted step before it (0: none, read as 1).
inline double pi_next_dt(double dt, double E, double E_prev, double error_order, const Params3& p)
{
    const double k = error_order + 1;
    const double ep = E_prev > 0 ? E_prev : 1.0;
    double factor = 0.9 * std::pow(1.0 / E, 0.7 / k) * std::pow(ep, 0.4 / k);
    if (factor >= 10) factor = 10;
    else if (factor < 0.2) factor = 0.2;
    double next = dt * factor;
    if (next < p.min_stepsize) next = p.min_stepsize;
    else if (next > p.max_stepsize) next = p.max_stepsize;
    return next;
}

inline void loop_init(LoopState& st, const Params3& p)
{
    st.dt = p.max_stepsize;                      // simulation.hpp:1167
    st.nb = build_neighbors(st.cells, p);   // :1277
    st.rebuilds = 1;
}

// One iteration of `while (!terminate)`; `cc_once` evaluates the stage-
// invariant pair forces once per attempt instead of once per stage.
inline void loop_iteration(LoopState& st, const Params3& p, bool cc_once = false)
{
    std::vector<int> to_divide(st.cells.n);
    int ndiv = 0;
    for (int i = 0; i < st.cells.n; ++i) { to_divide[i] = st.cells(i, C_L) > p.Ldiv; ndiv += to_divide[i]; }
    const int n_before = st.cells.n;
    st.cells = divide_cells(st.cells, st.parents, st.t, p, to_divide, st.iter);
    if (ndiv > 0)
    {
        st.divisions += ndiv;
        // simulation.hpp:1650-1656: daughters (mother's row, appended row) may switch group
        if (p.switch_mode == 2 && st.cells.n >= p.n_cells_start_switch)
        {
            std::vector<std::pair<int, int> > pairs;
            for (int i = 0, m = 0; i < n_before; ++i)
                if (to_divide[i]) pairs.push_back(std::make_pair(i, n_before + m++));
            switch_groups_inherit(st.cells, pairs, p, st.iter);
        }
        st.nb = build_neighbors(st.cells, p);
        st.rebuilds++;
    }
    if (p.integration_mode == 0)
    {
        // simulation.hpp:1279-1290, 1786-1798: one velocity-Verlet step at the fixed dt
        if (p.M0 <= 0) throw std::runtime_error("Initial cell mass must be defined when using velocity Verlet");
        const double rho = p.M0 / (PI * ((4. / 3.) * std::pow(p.R, 3) + p.R * p.R * p.L0));
        st.cells = step_velocity_verlet(st.cells, st.nb, st.dt, p, rho, st.iter);
        st.attempts++;
        st.last_max_error = 0;
    }
    else
    {
        const Tableau tab = make_tableau(p.integration_mode);
        Arr6 errors;
        int attempt = 0;
        Cells cn = step_rk_adaptive(tab, st.cells, st.nb, st.dt, p, st.iter, attempt++, errors, cc_once);
        st.attempts++;
        double max_error = max_scaled_error(st.cells, errors, p.max_error_allowed, p.min_error);
        const bool proposal = p.controller == 2;
        if (max_error > 1.0) st.rejected++;
        if (proposal && !(max_error > 1.0))
        {
            // the PI proposal passed the error test: it is the accepted step
        }
        else if (proposal || st.iter % p.iter_update_stepsize == 0)
        {
            bool exceeded = (max_error > 1.0);
            double q1 = 1.0 / (tab.error_order + 1);
            double factor = 0.9 * std::pow(1.0 / max_error, q1);
            if (factor >= 10) factor = 10;
            else if (factor < 0.2) factor = 0.2;
            int j = 0;
            while (exceeded && j < p.max_tries_update_stepsize)
            {
                double dt_new = st.dt * factor;
                cn = step_rk_adaptive(tab, st.cells, st.nb, dt_new, p, st.iter, attempt++, errors, cc_once);
                st.attempts++;
                max_error = max_scaled_error(st.cells, errors, p.max_error_allowed, p.min_error);
                exceeded = (max_error > 1.0);
                factor *= 0.9 * std::pow(1.0 / max_error, q1);
                if (factor >= 10) { factor = 10; break; }
                else if (factor < 0.2) { factor = 0.2; break; }
                j++;
            }
            if (st.dt * factor < p.min_stepsize) factor = p.min_stepsize / st.dt;
            else if (st.dt * factor > p.max_stepsize) factor = p.max_stepsize / st.dt;
            st.dt *= factor;
            cn = step_rk_adaptive(tab, st.cells, st.nb, st.dt, p, st.iter, attempt++, errors, cc_once);
            st.attempts++;
            max_error = max_scaled_error(st.cells, errors, p.max_error_allowed, p.min_error);
        }
        st.prev_accepted_error = st.last_max_error;
        st.last_max_error = max_error;
        st.cells = cn;
    }
    const double dt_accepted = st.dt;
    grow_cells(st.cells, st.dt, p.R);
    update_neighbor_distances(st.cells, st.nb);
    if (!p.no_surface && p.basal_only && basal_compact(st.cells, p) > 0)
    {
        st.nb = build_neighbors(st.cells, p);
        st.rebuilds++;
    }
    st.t += st.dt;
    st.iter++;
    if (st.iter % p.iter_update_neighbors == 0)
    {
        st.nb = build_neighbors(st.cells, p);
        st.rebuilds++;
    }
    // simulation.hpp:1866-2022.  The reference compares its cell count from before the
    // basal compaction here (and loops over that many cells); the current count is used.
    if (p.switch_mode == 1 && st.cells.n >= p.n_cells_start_switch)
        switch_groups_markov(st.cells, p, st.dt, st.iter);
    if (p.switch_mode != 0)
    {
        ramp_attributes(st.cells, p, st.dt);
        if (p.adhesion_mode != 0)
        {
            ramp_gamma(st.cells, p, st.dt);
            if (p.modulate_local_viscosity) modulate_viscosity(st.cells, st.nb, p);
        }
    }
    // the PI proposal for the next step, once this step's dt has served the ramps
    if (p.controller == 2 && p.integration_mode != 0)
        st.dt = pi_next_dt(dt_accepted, st.last_max_error, st.prev_accepted_error,
                           make_tableau(p.integration_mode).error_order, p);
}

}   // namespace oracle
