// Velocity-Verlet step of the 3-D model (integration mode 0; kmnam/biofilm-ABMs,
// ABM-3d/ABM-3d-cpp/include: stepVelocityVerlet, mechanics.hpp:2668-2996, called from
// simulation.hpp:1786-1798 with the cell density of simulation.hpp:1279-1290):
//
//   k_verlet_pairs  (y0)       the pair forces in their include_constraint form
//   k_verlet_cells  phase 0    forces -> accelerations, half kick, drift of both cell ends
//                              with the half-step velocity and angular velocity -> geom_c
//   k_verlet_pairs  (drifted)  the same at the drifted state (updateNeighborDistances)
//   k_verlet_cells  phase 1    forces -> second half kick, dn = omega x n, growth
//   k_verlet_accept            the clock and the loop's counters
//
// The include_constraint forms (mechanics.hpp:1298-1311, 1554-1566, 1608-1617,
// adhesion.hpp:355-366, mechanics.hpp:718-755, 845-886, 1152-1161): the orientation rows of
// the Hertz, hard-core and friction terms become (s n) x v; those of the JKR term become
// s (v - (n . v) n); the surface terms trade their nz row for x, y torques.  Both are linear
// in the pair's share v and the body coordinate s, so a pair records its share v, s and the
// JKR part of v, and each cell applies n x and the projection to the sums over its row.
// The forces of one half step (mechanics.hpp:2834-2862, 2919-2947): the conservative forces,
// plus the noise, minus the ambient viscosity eta0 l^3 (dr, l^6 (n x dn) / 12)
// (mechanics.hpp:1784-1820), minus the cell-surface friction (mechanics.hpp:1821-1917),
// capped row by row at cell_surface_coulomb_coeff times the constrained surface repulsion.
#include "abm_kernels.cuh"
#include "abm_pair.cuh"

namespace abm {

const int VV_T = 256;

static inline int cdiv_v(int a, int b) { return (a + b - 1) / b; }

// include_constraint form of one pair's shares at the given state (geom, vel): (v, s)
// into both entries as the Runge-Kutta pass writes them, and the JKR part of v into pbuf
__global__ void k_verlet_pairs(const Geom* __restrict__ geom, const Vel* __restrict__ vel,
                               const int4* __restrict__ pairs, const Ctrl* ctrl, ForceParams fp,
                               const double* __restrict__ td, const double* __restrict__ tr, double4* jbuf,
                               double4* pbuf)
{
    if (ctrl->halted) return;
    const int n_pairs = ctrl->n_dir >> 1;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_pairs; q += gridDim.x * blockDim.x)
    {
        const int4 pr = pairs[q];
        const Geom gi = load_geom(geom, pr.x), gj = load_geom(geom, pr.y);
        const PairOut p = pair_force_fp64(gi, gj, fp, td, tr);
        double4 own = make_double4(0.0, 0.0, 0.0, 0.0), other = own, part = own;
        if (p.touch)
        {
            own = make_double4(p.vx, p.vy, p.vz, p.s);
            other = make_double4(p.vx, p.vy, p.vz, p.t);
            const double ux = p.dx / p.dist, uy = p.dy / p.dist, uz = p.dz / p.dist;
            part = make_double4(p.mj * ux, p.mj * uy, p.mj * uz, 0.0);
            if (fp.fric)
            {
                // mechanics.hpp:1031-1175 at this state: the stored velocities of the state
                // and the planar decision of its contact points
                const X3 dv = x3(p.dx, p.dy, p.dz);
                const Vel ui = vel[pr.x], uj = vel[pr.y];
                const double eta = fmin(fp.feta[pr.x], fp.feta[pr.y]);
                double rv[3];
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    rv[c] = (ui.v[c] + p.s * ui.v[3 + c]) - (uj.v[c] + p.t * uj.v[3 + c]);
                bool flat = false;
                if (fp.surface && fabs(__ddiv_rn(p.dz, p.dist)) < 1e-3)
                {
                    const double lim = 1.01 * fp.R;
                    flat = __dadd_rn(gi.rz, __dmul_rn(p.s, gi.nz)) < lim &&
                           __dadd_rn(gj.rz, __dmul_rn(p.t, gj.nz)) < lim;
                }
                double f[3];
                friction_force(dv, p.dist, flat, rv, eta, fp, f);
                own.x -= f[0]; own.y -= f[1]; own.z -= f[2];
                other.x -= f[0]; other.y -= f[1]; other.z -= f[2];
            }
        }
        jbuf[pr.z] = own;
        jbuf[pr.w] = other;
        pbuf[pr.z] = part;
        pbuf[pr.w] = part;
    }
}

struct VerletArgs {
    const Geom* g_in;        // the state the forces are evaluated at
    const Vel* v_in;
    Geom* g_out;             // phase 0: the drifted state; phase 1: the new state
    Vel* v_out;
    Phys* phys;
    double4* whalf;          // half-step angular velocity of each cell
    const int* row_ptr;
    const int* lower_end;
    const double4* jbuf;
    const double4* pbuf;
    double rho;              // cell density M0 / (pi ((4/3) R^3 + R^2 L0))
};

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// the generalised force of one half step on cell i at state (g, u); writes f[6]
__device__ __forceinline__ void verlet_force(const StepParams& sp, const VerletArgs& a, int i, const Geom& g,
                                             const Vel& u, const Phys& ph, int iter, double f[6])
{
    const MechParams& P = sp.mp;
    const double n[3] = {g.nx, g.ny, g.nz};
    // the pair sums in CSR order, then the constrained orientation rows
    double F[3] = {0, 0, 0}, Tc[3] = {0, 0, 0}, Tp[3] = {0, 0, 0};
    const int le = a.lower_end[i], r1 = a.row_ptr[i + 1];
    for (int e = a.row_ptr[i]; e < r1; ++e)
    {
        const double4 js = a.jbuf[e], pp = a.pbuf[e];
        const double sg = e < le ? 1.0 : -1.0, w = sg * js.w;
        F[0] += sg * js.x; F[1] += sg * js.y; F[2] += sg * js.z;
        Tc[0] += w * (js.x - pp.x); Tc[1] += w * (js.y - pp.y); Tc[2] += w * (js.z - pp.z);
        Tp[0] += w * pp.x; Tp[1] += w * pp.y; Tp[2] += w * pp.z;
    }
    double dE[6];
    double tcr[3];
    cross3(n, Tc, tcr);
    const double np = (n[0] * Tp[0] + n[1] * Tp[1]) + n[2] * Tp[2];
    dE[0] = F[0]; dE[1] = F[1]; dE[2] = F[2];
    dE[3] = tcr[0] + (Tp[0] - np * n[0]);
    dE[4] = tcr[1] + (Tp[1] - np * n[1]);
    dE[5] = tcr[2] + (Tp[2] - np * n[2]);
    // cell-surface repulsion and adhesion, include_constraint (mechanics.hpp:673-910)
    double rep[6] = {0, 0, 0, 0, 0, 0}, adh[6] = {0, 0, 0, 0, 0, 0};
    const bool a2 = g.nz < P.nz_threshold;
    const double l = ph.l, h = g.h, R = P.R;
    double ss = 0.0;
    EndPow w;
    w.p = w.q = w.sp = w.sq = 0.0;
    if (!P.no_surface)
    {
        if (a2) surface_dEdq_flat(P, g.rz, l, ph.sigma0, rep[2], adh[2]);
        else
        {
            ss = (R - g.rz) / g.nz;
            w = end_pows(g.rz, g.nz, R, h, ss);
            const double nz = g.nz, nz2 = nz * nz, inz = 1.0 / nz;
            const double pf0 = 2 * P.E0;
            rep[2] = -pf0 * ((1.0 - nz2) * integral1(w, inz, h, 4, ss) + P.sqrtR * nz2 * integral1(w, inz, h, 3, ss));
            const double cx = g.ny, cy = -g.nx;
            const double W = (1.0 - nz2) * integral2(w, inz, h, 4, ss) + P.sqrtR * nz2 * integral2(w, inz, h, 3, ss);
            rep[3] = -pf0 * cx * W;
            rep[4] = -pf0 * cy * W;
            const double a0 = P.sqrtR / 2, a1 = 2 * M_PI * R;
            const bool partial = fabs(ss) < h;
            const double term2 = partial ? (a1 / 2) * nz : 0.0;
            adh[2] = (a0 * (1 - nz2) * integral1(w, inz, h, 1, ss) + term2) * ph.sigma0;
            const double i2 = integral2(w, inz, h, 1, ss);
            const double w1 = partial ? (a1 / 2) * ss * nz * cx : 0.0;
            const double w2 = partial ? (a1 / 2) * ss * nz * cy : 0.0;
            adh[3] = (a0 * (1 - nz2) * i2 * cx - w1) * ph.sigma0;
            adh[4] = (a0 * (1 - nz2) * i2 * cy - w2) * ph.sigma0;
        }
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) f[c] = ((-dE[c]) - rep[c]) - adh[c];
    if (sp.noise_on)
    {
        // the attempt-0 noise of the iteration (sample_noise of the step), as the
        // Runge-Kutta path draws it
        for (int k = 0; k < 3; ++k)
        {
            uint32_t x[4] = {(uint32_t)iter, 0u, (uint32_t)i, (uint32_t)k};
            philox4x32_10(x, (uint32_t)sp.seed, (uint32_t)(sp.seed >> 32) ^ RNG_PURPOSE_NOISE);
            const double u0 = philox_u01(x[0], x[1]), u1 = philox_u01(x[2], x[3]);
            f[2 * k] += -sp.noise_max[2 * k] + 2 * sp.noise_max[2 * k] * u0;
            f[2 * k + 1] += -sp.noise_max[2 * k + 1] + 2 * sp.noise_max[2 * k + 1] * u1;
        }
    }
    // ambient viscosity (mechanics.hpp:1784-1820)
    const double dn[3] = {u.v[3], u.v[4], u.v[5]};
    double om[3];
    cross3(n, dn, om);
    const double li = pow(l, 3.0);
    const double A = ph.eta0 * li, B = ph.eta0 * li * li * li;
    f[0] -= A * u.v[0]; f[1] -= A * u.v[1]; f[2] -= A * u.v[2];
    f[3] -= B * om[0] / 12; f[4] -= B * om[1] / 12; f[5] -= B * om[2] / 12;
    if (!P.no_surface)
    {
        // cell-surface friction (mechanics.hpp:1821-1917)
        double csf[6] = {0, 0, 0, 0, 0, 0};
        const double q[3] = {u.v[0], u.v[1], 0.0};
        const double m[3] = {om[1] * n[2] - om[2] * n[1], om[2] * n[0] - om[0] * n[2], 0.0};
        const double eta = ph.eta1;
        if (a2)
        {
            const double phz = R - g.rz;
            if (phz > 0)
            {
                const double area = sqrt(R) * sqrt(phz) * l;
                csf[0] = eta * q[0] * area / R;
                csf[1] = eta * q[1] * area / R;
                const double cz = n[0] * m[1] - n[1] * m[0];
                csf[5] = eta * cz * area * (l * l) / (12 * R);
            }
        }
        else
        {
            double A1, A2, A3;
            area_integrals(P, g.nz, h, ss, w, A1, A2, A3);
            csf[0] = eta * (q[0] * A1 + m[0] * A2) / R;
            csf[1] = eta * (q[1] * A1 + m[1] * A2) / R;
            double c1[3], c2[3];
            cross3(n, q, c1);
            cross3(n, m, c2);
            csf[3] = eta * (c1[0] * A2 + c2[0] * A3) / R;
            csf[4] = eta * (c1[1] * A2 + c2[1] * A3) / R;
            csf[5] = eta * (c1[2] * A2 + c2[2] * A3) / R;
        }
        if (P.coulomb > 0)
        {
            double sf = 0, sr = 0;
            for (int c = 0; c < 6; ++c) { sf += csf[c] * csf[c]; sr += rep[c] * rep[c]; }
            const double fn = sqrt(sf), max_norm = P.coulomb * sqrt(sr);
            if (fn > max_norm)
                for (int c = 0; c < 6; ++c) csf[c] *= (max_norm / fn);
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) f[c] -= csf[c];
    }
}

// accelerations (mechanics.hpp:2863-2877): forces over the mass, the torque split along n
// and across it over the two moments of inertia of a capsule of density rho
__device__ __forceinline__ void verlet_accel(const double f[6], const double n[3], double length, double rho,
                                             double R, double lin[3], double ang[3])
{
    const double volume = M_PI * ((4. / 3.) * pow(R, 3.0) + R * R * length);
    const double mass = rho * volume;
    const double diam = 2 * R, d2 = diam * diam, d3 = d2 * diam, d4 = d3 * diam;
    const double l2 = length * length, l3 = l2 * length;
    const double mom_par = d4 * (length / 32 + diam / 60) * (rho * M_PI);
    const double mom_perp = d2 * (4 * d3 + 15 * length * d2 + 20 * l2 * diam + 10 * l3) / 480 * (rho * M_PI);
    const double tq[3] = {f[3], f[4], f[5]};
    const double tn = (tq[0] * n[0] + tq[1] * n[1]) + tq[2] * n[2];
    for (int c = 0; c < 3; ++c)
    {
        lin[c] = f[c] / mass;
        const double tpar = tn * n[c], tperp = tq[c] - tpar;
        ang[c] = tpar / mom_par + tperp / mom_perp;
    }
}

__device__ __forceinline__ void normalize3(double n[3])
{
    const double nrm = sqrt((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2]);
    n[0] /= nrm; n[1] /= nrm; n[2] /= nrm;
    if (n[2] < 0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
}

template <int PHASE>
__global__ void k_verlet_cells(Ctrl* ctrl, StepParams sp, VerletArgs a)
{
    if (ctrl->halted) return;
    const int n = ctrl->n;
    const double dt = ctrl->dt, hdt = 0.5 * dt;
    const int iter = ctrl->iter;
    const double R = sp.mp.R;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const Geom g = a.g_in[i];
        const Vel u = a.v_in[i];
        const Phys ph = a.phys[i];
        double f[6];
        verlet_force(sp, a, i, g, u, ph, iter, f);
        const double nv[3] = {g.nx, g.ny, g.nz};
        double lin[3], ang[3];
        verlet_accel(f, nv, ph.l, a.rho, R, lin, ang);
        Geom go = g;
        Vel vo;
        if (PHASE == 0)
        {
            // half kick, then the two ends drift with v and the rotation w x (p - q) / 2
            const double dn[3] = {u.v[3], u.v[4], u.v[5]};
            double om[3];
            cross3(nv, dn, om);
            double vi[3], wi[3];
            for (int c = 0; c < 3; ++c) { vi[c] = u.v[c] + hdt * lin[c]; wi[c] = om[c] + hdt * ang[c]; }
            const double r[3] = {g.rx, g.ry, g.rz};
            double p[3], q[3], pq[3];
            for (int c = 0; c < 3; ++c) { p[c] = r[c] - g.h * nv[c]; q[c] = r[c] + g.h * nv[c]; pq[c] = p[c] - q[c]; }
            double cw[3];
            cross3(wi, pq, cw);
            double pn[3], qn[3], rn[3], nn[3];
            for (int c = 0; c < 3; ++c)
            {
                const double half = cw[c] / 2;
                pn[c] = p[c] + dt * (vi[c] + half);
                qn[c] = q[c] + dt * (vi[c] - half);
                rn[c] = (pn[c] + qn[c]) / 2;
                nn[c] = (qn[c] - pn[c]) / ph.l;
            }
            double dni[3];
            cross3(wi, nv, dni);
            normalize3(nn);
            go.rx = rn[0]; go.ry = rn[1]; go.rz = rn[2];
            go.nx = nn[0]; go.ny = nn[1]; go.nz = nn[2];
            for (int c = 0; c < 3; ++c) { vo.v[c] = vi[c]; vo.v[3 + c] = dni[c]; }
            a.whalf[i] = make_double4(wi[0], wi[1], wi[2], 0.0);
        }
        else
        {
            // second half kick at the drifted state, dn = w x n, then growCells
            // (growth.hpp:51-57) with the step's dt
            const double4 wh = a.whalf[i];
            const double wf[3] = {wh.x + hdt * ang[0], wh.y + hdt * ang[1], wh.z + hdt * ang[2]};
            double dni[3];
            cross3(wf, nv, dni);
            for (int c = 0; c < 3; ++c) { vo.v[c] = u.v[c] + hdt * lin[c]; vo.v[3 + c] = dni[c]; }
            double nn[3] = {g.nx, g.ny, g.nz};
            normalize3(nn);
            go.nx = nn[0]; go.ny = nn[1]; go.nz = nn[2];
            const double lg = ph.l + ph.growth * (4 * R / 3 + ph.l) * dt;
            go.h = lg / 2;
            a.phys[i].l = lg;
            if (!(isfinite(go.rx) && isfinite(go.ry) && isfinite(go.rz) && isfinite(nn[0]) && isfinite(nn[1]) &&
                  isfinite(nn[2])))
                atomicOr(&ctrl->status, (int)ST_NAN);
        }
        a.g_out[i] = go;
        a.v_out[i] = vo;
    }
}

// the accepted step's bookkeeping (the accepted branch of the controller, with the
// reference's zero error for a Verlet step, simulation.hpp:1786-1798)
__global__ void k_verlet_accept(Ctrl* c)
{
    if (c->halted) return;
    c->attempts += 1;
    c->last_max_error = 0.0;
    const int h = c->hist_pos;
    c->hist_dt[h] = c->dt;
    c->hist_err[h] = 0.0;
    c->hist_acc[h] = 1;
    c->hist_pos = (h + 1) % HIST;
    c->since_div = c->n_divide > 0 ? 0 : c->since_div + 1;
    c->cell_steps += c->n;
    c->t += c->dt;
    c->iter += 1;
    c->iterations += 1;
    if (c->dt_write > 0)
    {
        const double t_old_factor = fmod(c->t - c->dt + 1e-12, c->dt_write);
        const double t_new_factor = fmod(c->t + 1e-12, c->dt_write);
        if (t_old_factor > t_new_factor) c->frame_due = 1;
    }
    c->screen_valid = 0;
}

void launch_verlet_step(Geom* geom, Vel* vel, Phys* phys, Geom* geom_c, Vel* vel_c, double4* whalf, Ctrl* ctrl,
                        const StepParams& sp, const ForceParams& fp, const double* td, const double* tr,
                        const int4* pairs, const int* row_ptr, const int* lower_end, double4* jbuf, double4* pbuf,
                        double rho, int cap_cells, int cap_pairs, cudaStream_t st)
{
    const int pb = max(min(cdiv_v(cap_pairs, VV_T), 148 * 16), 1);
    const int cb = max(min(cdiv_v(cap_cells, VV_T), 148 * 8), 1);
    VerletArgs a0 = {geom, vel, geom_c, vel_c, phys, whalf, row_ptr, lower_end, jbuf, pbuf, rho};
    VerletArgs a1 = {geom_c, vel_c, geom, vel, phys, whalf, row_ptr, lower_end, jbuf, pbuf, rho};
    k_verlet_pairs<<<pb, VV_T, 0, st>>>(geom, vel, pairs, ctrl, fp, td, tr, jbuf, pbuf);
    k_verlet_cells<0><<<cb, VV_T, 0, st>>>(ctrl, sp, a0);
    k_verlet_pairs<<<pb, VV_T, 0, st>>>(geom_c, vel_c, pairs, ctrl, fp, td, tr, jbuf, pbuf);
    k_verlet_cells<1><<<cb, VV_T, 0, st>>>(ctrl, sp, a1);
    k_verlet_accept<<<1, 1, 0, st>>>(ctrl);
}

}   // namespace abm
