// ORACLE — test infrastructure only.  A plain C++17 restatement of the 2-D
// mechanics step of kmnam/biofilm-ABMs (ABM-2d/ABM-2d-cpp), against which tests/
// compare the 2-D CUDA path.  The product library never links, includes
// or calls anything under oracle/.
//
// Geometry is shared with the 3-D restatement (abm3d.hpp): the 2-D reference
// builds its segments as CGAL Segment_3 with z = 0 (2D/include/distances.hpp:
// 63-83) and runs the same distBetweenCells algorithm on two components
// (2D/include/distances.hpp:199-350), so distances, the neighbor table and the
// division room checks are taken from the 3-D functions on cells embedded with
// z = 0 and nz = 0 (every product with a zero component is an exact zero, so
// each sum and norm rounds as in two components).  The 2-D daughter rotation
// (2D/include/utils.hpp:374-380) is rotateXY with z = 0 followed by an
// out-of-plane rotation by 0, which returns its input unchanged.
//
// Forces, velocities, the RK step and the controller are restated from the 2-D
// files directly.  Random draws follow the counter policy of philox.hpp.
#pragma once
#include "abm3d.hpp"

namespace oracle {

// ABM-2d/ABM-2d-cpp/include/indices.hpp:17-41
enum Col2 {
    D_ID = 0, D_RX = 1, D_RY = 2, D_NX = 3, D_NY = 4, D_DRX = 5, D_DRY = 6, D_DNX = 7, D_DNY = 8,
    D_L = 9, D_HALF_L = 10, D_T0 = 11, D_GROWTH = 12, D_ETA0 = 13, D_ETA1 = 14, D_MAXETA1 = 15, D_GROUP = 16
};
const int NCOLS_2D = 17;

struct Params2 {
    double R = 0.8, Rcell = 0.5, E0 = 3900.0, Ecell = 3.9e6;
    double sigma0 = 100.0;                 // cell-surface adhesion energy density (rho_c)
    double Ldiv = 5.6, neighbor_threshold = 3.6;
    int adhesion_mode = 0;                 // 0 NONE, 1 JKR (2D/include/mechanics.hpp:51-57)
    double adhesion_strength = 0, adhesion_mindist = 0;
    int integration_mode = 2;              // 2-D driver: Bogacki-Shampine 3(2)
    double max_stepsize = 1e-6, min_stepsize = 1e-9;
    double max_error_allowed = 1e-8, min_error = 1e-30;
    int max_tries_update_stepsize = 3;
    int iter_update_stepsize = 1, iter_update_neighbors = 100;
    double max_noise = 0;
    double growth_mean = 0, growth_std = 0, daughter_length_std = 0, daughter_angle_bound = 0;
    uint64_t rng_seed = 42;
    // explicit cellCellRepulsiveForces prefactors (the reference's unit tests pass
    // their own, 2D/test/src/testHertz.cpp:201-204); unused when use_pf == 0
    int use_pf = 0;
    double pf[3] = {0, 0, 0};
    RngStream* stream = nullptr;           // the reference's sequential source (abm3d.hpp), or Philox
};

// 2D/include/simulation.hpp:232-235 (the code's exponents: 0.5, 2.5 and 0.5)
inline void prefactors_2d(const Params2& p, double pf[3])
{
    if (p.use_pf) { pf[0] = p.pf[0]; pf[1] = p.pf[1]; pf[2] = p.pf[2]; return; }
    pf[0] = 2.5 * p.E0 * std::sqrt(p.R);
    pf[1] = 2.5 * p.E0 * std::sqrt(p.R) * std::pow(2 * (p.R - p.Rcell), 2.5);
    pf[2] = 2.5 * p.Ecell * std::sqrt(p.Rcell);
}

// 2D/include/simulation.hpp:237
inline double surface_contact_density(const Params2& p)
{
    return std::pow(p.sigma0 * p.R * p.R / (4 * p.E0), 1. / 3.);
}

// 2-D cells in the 3-D layout (z = 0, nz = 0); maxeta1 rides in the sigma0 column
inline Cells embed3(const Cells& c)
{
    Cells e(c.n, NCOLS_REQUIRED_3D);
    for (int i = 0; i < c.n; ++i)
    {
        e(i, C_ID) = c(i, D_ID);
        e(i, C_RX) = c(i, D_RX); e(i, C_RY) = c(i, D_RY); e(i, C_RZ) = 0;
        e(i, C_NX) = c(i, D_NX); e(i, C_NY) = c(i, D_NY); e(i, C_NZ) = 0;
        e(i, C_DRX) = c(i, D_DRX); e(i, C_DRY) = c(i, D_DRY); e(i, C_DRZ) = 0;
        e(i, C_DNX) = c(i, D_DNX); e(i, C_DNY) = c(i, D_DNY); e(i, C_DNZ) = 0;
        e(i, C_L) = c(i, D_L); e(i, C_HALF_L) = c(i, D_HALF_L); e(i, C_T0) = c(i, D_T0);
        e(i, C_GROWTH) = c(i, D_GROWTH); e(i, C_ETA0) = c(i, D_ETA0); e(i, C_ETA1) = c(i, D_ETA1);
        e(i, C_SIGMA0) = c(i, D_MAXETA1); e(i, C_GROUP) = c(i, D_GROUP);
    }
    return e;
}

inline Cells extract2(const Cells& e, int ncols)
{
    Cells c(e.n, ncols);
    for (int i = 0; i < e.n; ++i)
    {
        c(i, D_ID) = e(i, C_ID);
        c(i, D_RX) = e(i, C_RX); c(i, D_RY) = e(i, C_RY);
        c(i, D_NX) = e(i, C_NX); c(i, D_NY) = e(i, C_NY);
        c(i, D_DRX) = e(i, C_DRX); c(i, D_DRY) = e(i, C_DRY);
        c(i, D_DNX) = e(i, C_DNX); c(i, D_DNY) = e(i, C_DNY);
        c(i, D_L) = e(i, C_L); c(i, D_HALF_L) = e(i, C_HALF_L); c(i, D_T0) = e(i, C_T0);
        c(i, D_GROWTH) = e(i, C_GROWTH); c(i, D_ETA0) = e(i, C_ETA0); c(i, D_ETA1) = e(i, C_ETA1);
        c(i, D_MAXETA1) = e(i, C_SIGMA0); c(i, D_GROUP) = e(i, C_GROUP);
    }
    return c;
}

// ------------------------------------------------------------------------
// Neighbor table, row = (i, j, dx, dy, si, sj), plus to_adhere per row
// ------------------------------------------------------------------------
struct Neighbors2 {
    std::vector<int> i, j, adhere;
    std::vector<double> dx, dy, si, sj;
    int size() const { return (int)i.size(); }
};

inline double row_norm(const Neighbors2& nb, int k)
{
    return std::sqrt(nb.dx[k] * nb.dx[k] + nb.dy[k] * nb.dy[k]);
}

// 2D/include/simulation.hpp:242-258 (one group, the pair (0, 0) in the adhesion
// map when adhesion is on): adhere iff dist > R + Rcell and dist < 2R at build time
inline void set_adhere(Neighbors2& nb, const Params2& p)
{
    nb.adhere.assign(nb.size(), 0);
    for (int k = 0; k < nb.size(); ++k)
    {
        const double dist = row_norm(nb, k);
        nb.adhere[k] = (p.adhesion_mode != 0 && dist > p.R + p.Rcell && dist < 2 * p.R) ? 1 : 0;
    }
}

// 2D/include/mechanics.hpp:293-365 (getCellNeighbors)
inline Neighbors2 get_cell_neighbors_2d(const Cells& cells, const Params2& p)
{
    Neighbors nb3 = get_cell_neighbors(embed3(cells), p.neighbor_threshold, p.R, p.Ldiv);
    Neighbors2 nb;
    nb.i = nb3.i; nb.j = nb3.j; nb.dx = nb3.dx; nb.dy = nb3.dy; nb.si = nb3.si; nb.sj = nb3.sj;
    set_adhere(nb, p);
    return nb;
}

// 2D/include/mechanics.hpp:376-419 (updateNeighborDistances); to_adhere is kept
inline void update_neighbor_distances_2d(const Cells& cells, Neighbors2& nb)
{
    Cells e = embed3(cells);
    for (int k = 0; k < nb.size(); ++k)
    {
        DistResult res = dist_cells(e, nb.i[k], nb.j[k]);
        nb.dx[k] = res.d.x; nb.dy[k] = res.d.y; nb.si[k] = res.s; nb.sj[k] = res.t;
    }
}

typedef std::vector<double> Arr4;   // n x 4, column-major
inline double& A4(Arr4& a, int n, int i, int k) { return a[(size_t)k * n + i]; }
inline double A4c(const Arr4& a, int n, int i, int k) { return a[(size_t)k * n + i]; }

// 2D/include/mechanics.hpp:448-547 (cellCellRepulsiveForces)
inline Arr4 repulsive_forces_2d(const Cells& cells, const Neighbors2& nb, const Params2& p)
{
    const int n = cells.n;
    Arr4 dEdq((size_t)n * 4, 0.0);
    if (n == 1) return dEdq;
    double pf[3];
    prefactors_2d(p, pf);
    const double R = p.R, Rcell = p.Rcell;
    for (int k = 0; k < nb.size(); ++k)
    {
        const int i = nb.i[k], j = nb.j[k];
        const double mag = row_norm(nb, k);
        const double dirx = nb.dx[k] / mag, diry = nb.dy[k] / mag;
        const double overlap = 2 * R - mag;
        const double si = nb.si[k], sj = nb.sj[k];
        double prefactor = 0;
        if (overlap > 0 && overlap < 2 * (R - Rcell))
            prefactor = pf[0] * std::pow(overlap, 1.5);
        else if (overlap >= 2 * (R - Rcell))
        {
            double term = pf[2] * std::pow(overlap - 2 * (R - Rcell), 1.5);
            prefactor = pf[1] + term;
        }
        if (overlap > 0)
        {
            const double vx = prefactor * dirx, vy = prefactor * diry;
            const double nix = cells(i, D_NX), niy = cells(i, D_NY);
            const double njx = cells(j, D_NX), njy = cells(j, D_NY);
            const double wi = nix * vx + niy * vy;
            const double wj = njx * vx + njy * vy;
            A4(dEdq, n, i, 0) += vx; A4(dEdq, n, i, 1) += vy;
            A4(dEdq, n, i, 2) += si * (-wi * nix + vx); A4(dEdq, n, i, 3) += si * (-wi * niy + vy);
            A4(dEdq, n, j, 0) += -vx; A4(dEdq, n, j, 1) += -vy;
            A4(dEdq, n, j, 2) += sj * (wj * njx - vx); A4(dEdq, n, j, 3) += sj * (wj * njy - vy);
        }
    }
    return dEdq;
}

// 2D/include/mechanics.hpp:572-670 (cellCellAdhesiveForces, JKR mode) with
// 2D/include/adhesion.hpp:403-448 (forcesJKRLagrange, include_constraint = true)
inline Arr4 adhesive_forces_2d(const Cells& cells, const Neighbors2& nb, const Params2& p)
{
    const int n = cells.n;
    Arr4 dEdq((size_t)n * 4, 0.0);
    if (n == 1 || p.adhesion_mode == 0) return dEdq;
    const double R = p.R, strength = p.adhesion_strength, dmin = p.adhesion_mindist;
    for (int k = 0; k < nb.size(); ++k)
    {
        const double mag = row_norm(nb, k);
        const double overlap = 2 * R - mag;
        if (!(nb.adhere[k] && overlap > 0)) continue;
        const int i = nb.i[k], j = nb.j[k];
        const double dist = mag;
        double f[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
        if (dist <= 2 * R)
        {
            const double ux = nb.dx[k] / dist, uy = nb.dy[k] / dist;
            double term = PI * R;
            if (dist <= dmin) term *= (2 * R - dmin);
            else term *= (2 * R - dist);
            const double vx = term * ux, vy = term * uy;
            const double n1x = cells(i, D_NX), n1y = cells(i, D_NY), n2x = cells(j, D_NX), n2y = cells(j, D_NY);
            const double w1 = n1x * -vx + n1y * -vy;
            const double w2 = n2x * -vx + n2y * -vy;
            const double s = nb.si[k], t = nb.sj[k];
            f[0][0] = -vx; f[0][1] = -vy;
            f[1][0] = vx; f[1][1] = vy;
            f[0][2] = s * (-w1 * n1x - vx); f[0][3] = s * (-w1 * n1y - vy);
            f[1][2] = t * (w2 * n2x + vx); f[1][3] = t * (w2 * n2y + vy);
        }
        for (int c = 0; c < 4; ++c)
        {
            A4(dEdq, n, i, c) += strength * f[0][c];
            A4(dEdq, n, j, c) += strength * f[1][c];
        }
    }
    return dEdq;
}

// 2D/include/mechanics.hpp:264-279 (compositeViscosityForcePrefactors)
inline void viscosity_prefactors_2d(const Cells& cells, const Params2& p, std::vector<double>& K,
                                    std::vector<double>& L)
{
    const double rho = surface_contact_density(p);
    K.resize(cells.n); L.resize(cells.n);
    for (int i = 0; i < cells.n; ++i)
    {
        const double drag = cells(i, D_ETA0) + cells(i, D_ETA1) * rho / p.R;
        const double l = cells(i, D_L);
        K[i] = l * drag;
        L[i] = l * l * l * drag / 12;
    }
}

// Noise of one RK attempt: uniform on [-max, max] for (rx, ry, nx, ny)
// (2D/include/mechanics.hpp:1760-1771).  Counter policy shared with the 3-D
// path's draws of (rx, ry | rz, nx | ny, nz): rx, ry, nx, ny take the 3-D slots 0, 1, 3, 4.
inline Arr4 sample_noise_2d(int n, const Params2& p, int iter, int attempt)
{
    Arr4 noise((size_t)n * 4, 0.0);
    if (!(p.max_noise > 0)) return noise;
    if (p.stream)
    {
        // 2D/include/mechanics.hpp:1760-1771: four uniforms per cell, cell-major
        for (int i = 0; i < n; ++i)
            for (int c = 0; c < 4; ++c)
            {
                const double u = p.stream->uniform01();
                A4(noise, n, i, c) = -p.max_noise + 2 * p.max_noise * u;
            }
        return noise;
    }
    uint32_t k0, k1;
    rng_key(p.rng_seed, RNG_PURPOSE_NOISE, k0, k1);
    const double m = p.max_noise;
    for (int i = 0; i < n; ++i)
    {
        double u[6];
        for (int c = 0; c < 3; ++c)
        {
            Philox4 x = philox4x32_10((uint32_t)iter, (uint32_t)attempt, (uint32_t)i, (uint32_t)c, k0, k1);
            u[2 * c] = philox_u01(x.v[0], x.v[1]);
            u[2 * c + 1] = philox_u01(x.v[2], x.v[3]);
        }
        const int slot[4] = {0, 1, 3, 4};
        for (int c = 0; c < 4; ++c) A4(noise, n, i, c) = -m + 2 * m * u[slot[c]];
    }
    return noise;
}

// 2D/include/mechanics.hpp:1503-1667 (getVelocities) without confinement,
// cell-cell friction or the commented-out constraint projection
inline Arr4 get_velocities_2d(const Cells& cells, const Neighbors2& nb, const Params2& p, const Arr4& noise)
{
    const int n = cells.n;
    std::vector<double> K, L;
    viscosity_prefactors_2d(cells, p, K, L);
    Arr4 rep = repulsive_forces_2d(cells, nb, p);
    Arr4 adh = adhesive_forces_2d(cells, nb, p);
    Arr4 v((size_t)n * 4, 0.0);
    for (int i = 0; i < n; ++i)
    {
        double d[4];
        for (int c = 0; c < 4; ++c) d[c] = ((A4c(rep, n, i, c) + A4c(adh, n, i, c)) + 0.0) + A4c(noise, n, i, c);
        A4(v, n, i, 0) = -d[0] / K[i];
        A4(v, n, i, 1) = -d[1] / K[i];
        A4(v, n, i, 2) = -d[2] / L[i];
        A4(v, n, i, 3) = -d[3] / L[i];
    }
    return v;
}

// 2D/include/mechanics.hpp:1458-1465 (normalizeOrientations)
inline void normalize_orientations_2d(Cells& cells)
{
    for (int i = 0; i < cells.n; ++i)
    {
        const double nx = cells(i, D_NX), ny = cells(i, D_NY);
        const double norm = std::sqrt(nx * nx + ny * ny);
        cells(i, D_NX) = nx / norm;
        cells(i, D_NY) = ny / norm;
    }
}

// 2D/include/mechanics.hpp:1710-1817 (stepRungeKuttaAdaptive); errors is n x 4
inline Cells step_rk_2d(const Tableau& tab, const Cells& cells, const Neighbors2& nb, double dt,
                        const Params2& p, int iter, int attempt, Arr4& errors)
{
    const int n = cells.n;
    Arr4 noise = sample_noise_2d(n, p, iter, attempt);
    const int s = tab.s;
    std::vector<Arr4> vel;
    vel.push_back(get_velocities_2d(cells, nb, p, noise));
    for (int i = 1; i < s; ++i)
    {
        Arr4 mult((size_t)n * 4, 0.0);
        for (int j = 0; j < i; ++j)
            for (size_t k = 0; k < mult.size(); ++k) mult[k] += vel[j][k] * tab.a(i, j);
        Cells ci(cells);
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < n; ++r) ci(r, D_RX + c) += A4(mult, n, r, c) * dt;
        normalize_orientations_2d(ci);
        vel.push_back(get_velocities_2d(ci, nb, p, noise));
    }
    Cells cn(cells);
    Arr4 vf1((size_t)n * 4, 0.0), vf2((size_t)n * 4, 0.0);
    for (int i = 0; i < s; ++i)
        for (size_t k = 0; k < vf1.size(); ++k) { vf1[k] += vel[i][k] * tab.b[i]; vf2[k] += vel[i][k] * tab.bs[i]; }
    errors.assign((size_t)n * 4, 0.0);
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < n; ++r)
        {
            const double d1 = A4(vf1, n, r, c) * dt, d2 = A4(vf2, n, r, c) * dt;
            cn(r, D_RX + c) += d1;
            A4(errors, n, r, c) = d1 - d2;
        }
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < n; ++r) cn(r, D_DRX + c) = A4(vf1, n, r, c);
    normalize_orientations_2d(cn);
    return cn;
}

// 2D/include/simulation.hpp:645-650
inline double max_scaled_error_2d(const Cells& cells, const Arr4& errors, double tol, double min_error)
{
    const int n = cells.n;
    double mx = -std::numeric_limits<double>::infinity();
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < n; ++r)
        {
            const double z = 1.0 + std::fabs(cells(r, D_RX + c));
            const double v = A4c(errors, n, r, c) / (tol * z);
            if (v > mx) mx = v;
        }
    return std::max(mx, min_error);
}

// 2D/include/growth.hpp:51-56 (growCells)
inline void grow_cells_2d(Cells& cells, double dt, double R)
{
    for (int i = 0; i < cells.n; ++i)
    {
        cells(i, D_L) += cells(i, D_GROWTH) * (4 * R / 3 + cells(i, D_L)) * dt;
        cells(i, D_HALF_L) = cells(i, D_L) / 2;
    }
}

inline Params3 division_params(const Params2& p)
{
    Params3 q;
    q.R = p.R; q.Rcell = p.Rcell; q.Ldiv = p.Ldiv;
    q.growth_mean = p.growth_mean; q.growth_std = p.growth_std;
    q.daughter_length_std = p.daughter_length_std;
    q.daughter_angle_xy_bound = p.daughter_angle_bound;
    q.daughter_angle_z_bound = 0.0;
    q.rng_seed = p.rng_seed;
    q.stream = p.stream;
    q.planar_division = 1;
    return q;
}

// 2D/include/growth.hpp:166-436 (divideCells, one group): the 3-D restatement
// on the embedded cells with no out-of-plane angle (see the file header)
inline Cells divide_cells_2d(const Cells& cells, std::vector<int>& parents, double t, const Params2& p,
                             const std::vector<int>& to_divide, int iter, int* ntries_out = nullptr)
{
    Cells e = divide_cells(embed3(cells), parents, t, division_params(p), to_divide, iter, ntries_out);
    return extract2(e, cells.ncols);
}

// ------------------------------------------------------------------------
// Loop body (2D/include/simulation.hpp:549-774; switching, boundary, growth
// void, confinement and writing excluded)
// ------------------------------------------------------------------------
struct LoopState2 {
    Cells cells;
    Neighbors2 nb;
    std::vector<int> parents;
    double t = 0, dt = 0;
    int iter = 0;
    long long attempts = 0, rebuilds = 0, divisions = 0;
    double last_max_error = 0;
};

inline void loop_init_2d(LoopState2& st, const Params2& p)
{
    st.dt = p.max_stepsize;                       // 2D/include/simulation.hpp:212
    st.nb = get_cell_neighbors_2d(st.cells, p);   // :240
    st.rebuilds = 1;
}

inline void loop_iteration_2d(LoopState2& st, const Params2& p)
{
    const Tableau tab = make_tableau(p.integration_mode);
    std::vector<int> to_divide(st.cells.n);
    int ndiv = 0;
    for (int i = 0; i < st.cells.n; ++i) { to_divide[i] = st.cells(i, D_L) > p.Ldiv; ndiv += to_divide[i]; }
    st.cells = divide_cells_2d(st.cells, st.parents, st.t, p, to_divide, st.iter);
    if (ndiv > 0)
    {
        st.divisions += ndiv;
        st.nb = get_cell_neighbors_2d(st.cells, p);
        st.rebuilds++;
    }
    Arr4 errors;
    int attempt = 0;
    Cells cn = step_rk_2d(tab, st.cells, st.nb, st.dt, p, st.iter, attempt++, errors);
    st.attempts++;
    double max_error = max_scaled_error_2d(st.cells, errors, p.max_error_allowed, p.min_error);
    if (st.iter % p.iter_update_stepsize == 0)
    {
        bool exceeded = (max_error > 1.0);
        const double q1 = 1.0 / (tab.error_order + 1);
        double factor = 0.9 * std::pow(1.0 / max_error, q1);
        if (factor >= 10) factor = 10;
        else if (factor < 0.2) factor = 0.2;
        int j = 0;
        while (exceeded && j < p.max_tries_update_stepsize)
        {
            const double dt_new = st.dt * factor;
            cn = step_rk_2d(tab, st.cells, st.nb, dt_new, p, st.iter, attempt++, errors);
            st.attempts++;
            max_error = max_scaled_error_2d(st.cells, errors, p.max_error_allowed, p.min_error);
            exceeded = (max_error > 1.0);
            factor *= 0.9 * std::pow(1.0 / max_error, q1);
            if (factor >= 10) { factor = 10; break; }
            else if (factor < 0.2) { factor = 0.2; break; }
            j++;
        }
        if (st.dt * factor < p.min_stepsize) factor = p.min_stepsize / st.dt;
        else if (st.dt * factor > p.max_stepsize) factor = p.max_stepsize / st.dt;
        st.dt *= factor;
        cn = step_rk_2d(tab, st.cells, st.nb, st.dt, p, st.iter, attempt++, errors);
        st.attempts++;
        max_error = max_scaled_error_2d(st.cells, errors, p.max_error_allowed, p.min_error);
    }
    st.last_max_error = max_error;
    st.cells = cn;
    grow_cells_2d(st.cells, st.dt, p.R);
    update_neighbor_distances_2d(st.cells, st.nb);
    st.t += st.dt;
    st.iter++;
    if (st.iter % p.iter_update_neighbors == 0)
    {
        st.nb = get_cell_neighbors_2d(st.cells, p);
        st.rebuilds++;
    }
}

}   // namespace oracle
