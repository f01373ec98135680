// Pair force laws of the 3-D model shared by the Runge-Kutta pair pass and the
// velocity-Verlet step: Hertz repulsion, isotropic JKR adhesion from the fixed- or
// variable-gamma radius table, the hard-core term, and cell-cell kinetic friction
// (kmnam/biofilm-ABMs, ABM-3d/ABM-3d-cpp/include: mechanics.hpp, adhesion.hpp).
#pragma once
#include "abm_kernels.cuh"

namespace abm {

__device__ __forceinline__ double pow15(double x) { return x * sqrt(x); }

// adhesion.hpp:282-370: magnitude (term1 - term2) of the isotropic JKR force
// from the fixed-gamma radius table, overlap capped at max_overlap
__device__ __forceinline__ double jkr_magnitude(double dist, double gamma, const ForceParams& fp,
                                                const double* td, const double* tr)
{
    double delta = 2 * fp.R - dist;
    if (fp.max_overlap >= 0 && delta > fp.max_overlap) delta = fp.max_overlap;
    const int nm = fp.jkr_n;
    int k = (int)(delta / fp.jkr_step);
    k = k < 0 ? 0 : (k > nm - 2 ? nm - 2 : k);
    while (k > 0 && td[k] > delta) --k;
    while (k < nm - 2 && td[k + 1] <= delta) ++k;
    double d1 = td[k], d2 = td[k + 1], r1 = tr[k], r2 = tr[k + 1];
    double radius = (r1 * (d2 - delta) + r2 * (delta - d1)) / (d2 - d1);
    double Req = fp.R / 2;
    double a3 = radius * radius * radius;
    double term1 = 4 * fp.E0 * a3 / (3 * Req);
    double term2 = 4 * sqrt(M_PI * a3 * gamma * fp.E0);
    return term1 - term2;
}

// adhesion.hpp:412-526 (forcesIsotropicJKRLagrange with a variable-gamma table): the
// contact radius bilinearly interpolated on the cell of the (overlap, gamma) mesh that
// holds (delta, gamma), overlap capped at max_overlap; a gamma beyond the mesh takes
// the end cell.
template <class T>
__device__ __forceinline__ T jkr_radius_bilinear(T delta, T gamma, const ForceParams& fp, const double* td)
{
    const int nm = fp.jkr_n, ng = fp.jkr_ng;
    int k = (int)(delta / (T)fp.jkr_step);
    k = k < 0 ? 0 : (k > nm - 2 ? nm - 2 : k);
    while (k > 0 && (T)td[k] > delta) --k;
    while (k < nm - 2 && (T)td[k + 1] <= delta) ++k;
    int g = (int)(gamma / (T)fp.jkr_gstep);
    g = g < 0 ? 0 : (g > ng - 2 ? ng - 2 : g);
    while (g > 0 && (T)__ldg(fp.jkr_gam + g) > gamma) --g;
    while (g < ng - 2 && (T)__ldg(fp.jkr_gam + g + 1) <= gamma) ++g;
    const T d1 = (T)td[k], d2 = (T)td[k + 1];
    const T g1 = (T)__ldg(fp.jkr_gam + g), g2 = (T)__ldg(fp.jkr_gam + g + 1);
    const double* r = fp.jkr_rad2 + (size_t)k * ng + g;
    const T r11 = (T)__ldg(r), r12 = (T)__ldg(r + 1), r21 = (T)__ldg(r + ng), r22 = (T)__ldg(r + ng + 1);
    const T denom = (d2 - d1) * (g2 - g1);
    const T w11 = (d2 - delta) * (g2 - gamma) / denom;
    const T w12 = (d2 - delta) * (gamma - g1) / denom;
    const T w21 = (delta - d1) * (g2 - gamma) / denom;
    const T w22 = (delta - d1) * (gamma - g1) / denom;
    return ((w11 * r11 + w12 * r12) + w21 * r21) + w22 * r22;
}

__device__ __forceinline__ double jkr_magnitude_variable(double dist, double gamma, const ForceParams& fp,
                                                         const double* td)
{
    double delta = 2 * fp.R - dist;
    if (fp.max_overlap >= 0 && delta > fp.max_overlap) delta = fp.max_overlap;
    const double radius = jkr_radius_bilinear<double>(delta, gamma, fp, td);
    double Req = fp.R / 2;
    double a3 = radius * radius * radius;
    double term1 = 4 * fp.E0 * a3 / (3 * Req);
    double term2 = 4 * sqrt(M_PI * a3 * gamma * fp.E0);
    return term1 - term2;
}

// Force of one unordered pair (i > j, distance from cell i to cell j, as the
// reference's j < i loop computes it): magnitude m along d, returned as
// v = m d_hat with the body coordinates s (on i) and t (on j).  Cell i gains
// (v, s v) in dE/dq and cell j gains (-v, -t v) (mechanics.hpp:1390-1659).
struct PairOut { double vx, vy, vz, s, t, ovl; bool touch; double dx, dy, dz, dist, mj; };

__device__ __forceinline__ PairOut pair_force_fp64(const Geom& gi, const Geom& gj, const ForceParams& fp,
                                                   const double* td, const double* tr)
{
    PairOut out;
    out.touch = false;
    Dist d = dist_geom(gi, gj);
    double dist = xnorm(x3(d.dx, d.dy, d.dz));
    double overlap = 2 * fp.R - dist;
    if (!(overlap > 0)) return out;
    double ux = d.dx / dist, uy = d.dy / dist, uz = d.dz / dist;
    double m;
    double gamma = fp.adhesion ? fmin(gi.gamma, gj.gamma) : 0.0;
    out.mj = 0.0;
    if (fp.adhesion && gamma > 0)
    {
        m = fp.jkr_ng ? jkr_magnitude_variable(dist, gamma, fp, td) : jkr_magnitude(dist, gamma, fp, td, tr);
        out.mj = m;
    }
    else if (overlap <= fp.max_overlap) m = fp.pf0 * pow15(overlap);
    else
    {
        m = fp.pf2;
        if (!fp.adhesion) m += fp.pf1 * pow15(overlap - fp.max_overlap);
    }
    if (fp.adhesion && overlap > fp.max_overlap) m += fp.pf1 * pow15(overlap - fp.max_overlap);
    out.vx = m * ux; out.vy = m * uy; out.vz = m * uz;
    out.s = d.s; out.t = d.t; out.ovl = overlap; out.touch = true;
    out.dx = d.dx; out.dy = d.dy; out.dz = d.dz; out.dist = dist;
    return out;
}

// mechanics.hpp:1031-1175 (cellCellFrictionForces, include_constraint = false) for one
// touching pair (i, j), i = pr.x the larger index, from the pair's distance record: the
// friction force on cell i is -eta sqrt(Req overlap) times the tangential part of the
// relative velocity of the two contact points (dr + s dn of each cell's stored velocity),
// eta the smaller of the two coefficients, its norm capped at
// coulomb (4/3) E0 sqrt(Req) overlap^(3/2) when coulomb > 0.  A candidate contact
// (surface present, |dz / d| < 1e-3) whose contact points both lie below 1.01 R is taken
// in the xy-plane (distance, overlap and relative velocity without z).  Writes the force
// for both decisions (planar only for a candidate) and the decision at these positions.
__device__ __forceinline__ void friction_force(const X3 dv, double dist, bool planar, const double rv_in[3],
                                               double eta, const ForceParams& fp, double f[3])
{
    const double Req = fp.R / 2;
    X3 u;
    double overlap;
    double rv[3] = {rv_in[0], rv_in[1], rv_in[2]};
    if (planar)
    {
        const double d2 = xnorm(x3(dv.x, dv.y, 0.0));
        u = x3(dv.x / d2, dv.y / d2, 0.0);
        overlap = 2 * fp.R - d2;
        rv[2] = 0.0;
    }
    else
    {
        u = x3(dv.x / dist, dv.y / dist, dv.z / dist);
        overlap = 2 * fp.R - dist;
    }
    const double dd = (rv[0] * u.x + rv[1] * u.y) + rv[2] * u.z;
    const double c = -eta * sqrt(Req * overlap);
    f[0] = c * (rv[0] - dd * u.x);
    f[1] = c * (rv[1] - dd * u.y);
    f[2] = c * (rv[2] - dd * u.z);
    if (fp.coulomb_cc > 0)
    {
        const double fn = sqrt((f[0] * f[0] + f[1] * f[1]) + f[2] * f[2]);
        const double max_norm = fp.coulomb_cc * (4. / 3.) * fp.E0 * sqrt(Req) * pow(overlap, 1.5);
        if (fn > max_norm)
        {
            const double scale = max_norm / fn;
            f[0] *= scale; f[1] *= scale; f[2] *= scale;
        }
    }
}

}   // namespace abm
