// Host-side generator of seeded synthetic 3-D biofilm states (no CUDA).
//
// Sequential random placement on a uniform grid: each cell draws a centre
// uniform in a disk (radius disk_radius) with z uniform in [z_lo, z_hi], an
// azimuth uniform on [0, 2 pi), a polar angle from the substrate uniform on
// [0, pi/2] and a length uniform on [lmin, lmax]; with probability p_contact
// the centre is instead placed beside a random earlier cell at a centreline
// distance drawn uniformly in [min_gap, contact_dist) (an overlap inside the
// EPS shell).  A draw is rejected when any earlier cell lies closer than
// min_gap, so no pair overlaps into the cell cores.  Draws use SplitMix64.
#include <cmath>
#include <cstdint>
#include <vector>
#include <algorithm>

namespace {

struct SplitMix64 {
    uint64_t s;
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double u01() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
};

struct C3 { double x, y, z; };
inline C3 c3(double x, double y, double z) { C3 v = {x, y, z}; return v; }
inline C3 sub(C3 a, C3 b) { return c3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline C3 add(C3 a, C3 b) { return c3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline C3 mul(double s, C3 a) { return c3(s * a.x, s * a.y, s * a.z); }
inline double dot(C3 a, C3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double clamp01(double x) { return x < 0 ? 0 : (x > 1 ? 1 : x); }

// closest distance between two segments (Ericson 2005, sec. 5.1.9)
double seg_dist(C3 r1, C3 n1, double h1, C3 r2, C3 n2, double h2)
{
    C3 p1 = sub(r1, mul(h1, n1)), p2 = sub(r2, mul(h2, n2));
    C3 d1 = mul(2 * h1, n1), d2 = mul(2 * h2, n2), r = sub(p1, p2);
    double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r), c = dot(d1, r), b = dot(d1, d2);
    double denom = a * e - b * b;
    double s = denom > 1e-12 * a * e ? clamp01((b * f - c * e) / denom) : 0.0;
    double t = (b * s + f) / e;
    if (t < 0) { t = 0; s = clamp01(-c / a); }
    else if (t > 1) { t = 1; s = clamp01((b - c) / a); }
    C3 dv = sub(add(p2, mul(t, d2)), add(p1, mul(s, d1)));
    return std::sqrt(dot(dv, dv));
}

struct Grid3 {
    double x0, y0, z0, edge;
    int nx, ny, nz;
    std::vector<std::vector<int>> bins;
    int key(double x, double y, double z) const
    {
        int ix = std::min(std::max((int)std::floor((x - x0) / edge), 0), nx - 1);
        int iy = std::min(std::max((int)std::floor((y - y0) / edge), 0), ny - 1);
        int iz = std::min(std::max((int)std::floor((z - z0) / edge), 0), nz - 1);
        return (iz * ny + iy) * nx + ix;
    }
};

}   // namespace

// planar: every cell in the plane z = 0 with an in-plane orientation (the 2-D model);
// the draws are the same as in 3-D, with the out-of-plane components set to zero
static int generate(int n, unsigned long long seed, double disk_radius, double z_lo, double z_hi, double lmin,
                    double lmax, double min_gap, double contact_dist, double p_contact, int max_tries,
                    bool planar, double* out_r, double* out_n, double* out_l, int* placed)
{
    if (n <= 0 || !out_r || !out_n || !out_l) return -1;
    SplitMix64 rng = {seed * 0x2545F4914F6CDD1Dull + 1};
    Grid3 g;
    g.edge = min_gap + lmax;
    g.x0 = -disk_radius - g.edge; g.y0 = g.x0; g.z0 = std::min(z_lo, 0.0) - g.edge;
    g.nx = (int)std::ceil(2 * (disk_radius + g.edge) / g.edge) + 1;
    g.ny = g.nx;
    g.nz = (int)std::ceil((z_hi - g.z0 + g.edge) / g.edge) + 1;
    g.bins.assign((size_t)g.nx * g.ny * g.nz, std::vector<int>());
    std::vector<C3> R(n), N(n);
    std::vector<double> H(n);
    int count = 0;
    const double pi = 3.141592653589793238462643383279502884;
    for (int i = 0; i < n; ++i)
    {
        bool ok = false;
        for (int tr = 0; tr < max_tries && !ok; ++tr)
        {
            double az = 2 * pi * rng.u01(), pol = 0.5 * pi * rng.u01();
            if (planar) pol = 0.0;
            C3 nv = c3(std::cos(pol) * std::cos(az), std::cos(pol) * std::sin(az), planar ? 0.0 : std::sin(pol));
            double l = lmin + (lmax - lmin) * rng.u01();
            double h = l / 2;
            C3 rv;
            if (count > 0 && rng.u01() < p_contact)
            {
                int j = (int)(rng.u01() * count);
                double sj = (2 * rng.u01() - 1) * H[j];
                C3 u = c3(2 * rng.u01() - 1, 2 * rng.u01() - 1, 2 * rng.u01() - 1);
                if (planar) u.z = 0.0;
                u = sub(u, mul(dot(u, N[j]), N[j]));
                double un = std::sqrt(dot(u, u));
                if (un < 1e-9) continue;
                u = mul(1.0 / un, u);
                double dist = min_gap + (contact_dist - min_gap) * rng.u01();
                double si = (2 * rng.u01() - 1) * h;
                // centre so that the points r_j + sj n_j and r_i + si n_i are dist apart along u
                rv = sub(add(add(R[j], mul(sj, N[j])), mul(dist, u)), mul(si, nv));
                if (rv.z < z_lo || rv.z > z_hi || rv.x * rv.x + rv.y * rv.y > disk_radius * disk_radius)
                    continue;
            }
            else
            {
                double rad = disk_radius * std::sqrt(rng.u01()), ang = 2 * pi * rng.u01();
                rv = c3(rad * std::cos(ang), rad * std::sin(ang), z_lo + (z_hi - z_lo) * rng.u01());
                if (planar) rv.z = 0.0;
            }
            int k = g.key(rv.x, rv.y, rv.z);
            int iz = k / (g.nx * g.ny), iy = (k / g.nx) % g.ny, ix = k % g.nx;
            bool clash = false;
            for (int dz = -1; dz <= 1 && !clash; ++dz)
                for (int dy = -1; dy <= 1 && !clash; ++dy)
                    for (int dx = -1; dx <= 1 && !clash; ++dx)
                    {
                        int zz = iz + dz, yy = iy + dy, xx = ix + dx;
                        if (zz < 0 || yy < 0 || xx < 0 || zz >= g.nz || yy >= g.ny || xx >= g.nx) continue;
                        for (int j : g.bins[(size_t)(zz * g.ny + yy) * g.nx + xx])
                            if (seg_dist(rv, nv, h, R[j], N[j], H[j]) < min_gap) { clash = true; break; }
                    }
            if (clash) continue;
            R[count] = rv; N[count] = nv; H[count] = h;
            g.bins[k].push_back(count);
            out_r[3 * count] = rv.x; out_r[3 * count + 1] = rv.y; out_r[3 * count + 2] = rv.z;
            out_n[3 * count] = nv.x; out_n[3 * count + 1] = nv.y; out_n[3 * count + 2] = nv.z;
            out_l[count] = l;
            ++count;
            ok = true;
        }
    }
    if (placed) *placed = count;
    return count == n ? 0 : -3;
}

extern "C" int abm_generate_biofilm_3d(int n, unsigned long long seed, double disk_radius, double z_lo,
                                       double z_hi, double lmin, double lmax, double min_gap,
                                       double contact_dist, double p_contact, int max_tries,
                                       double* out_r, double* out_n, double* out_l, int* placed)
{
    return generate(n, seed, disk_radius, z_lo, z_hi, lmin, lmax, min_gap, contact_dist, p_contact, max_tries,
                    false, out_r, out_n, out_l, placed);
}

// 2-D colonies: centres uniform in a disk in the plane, orientations uniform in the plane
extern "C" int abm_generate_biofilm_2d(int n, unsigned long long seed, double disk_radius, double lmin,
                                       double lmax, double min_gap, double contact_dist, double p_contact,
                                       int max_tries, double* out_r, double* out_n, double* out_l, int* placed)
{
    return generate(n, seed, disk_radius, 0.0, 0.0, lmin, lmax, min_gap, contact_dist, p_contact, max_tries,
                    true, out_r, out_n, out_l, placed);
}

// Number of pairs closer than `dist` (segment distance), on the same grid.
extern "C" long long abm_count_close_pairs_3d(int n, const double* r, const double* nv, const double* l,
                                              double dist, double lmax)
{
    Grid3 g;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], r[3 * i + k]); hi[k] = std::max(hi[k], r[3 * i + k]); }
    g.edge = dist + lmax;
    g.x0 = lo[0]; g.y0 = lo[1]; g.z0 = lo[2];
    g.nx = (int)std::floor((hi[0] - lo[0]) / g.edge) + 1;
    g.ny = (int)std::floor((hi[1] - lo[1]) / g.edge) + 1;
    g.nz = (int)std::floor((hi[2] - lo[2]) / g.edge) + 1;
    g.bins.assign((size_t)g.nx * g.ny * g.nz, std::vector<int>());
    for (int i = 0; i < n; ++i) g.bins[g.key(r[3 * i], r[3 * i + 1], r[3 * i + 2])].push_back(i);
    long long cnt = 0;
    for (int i = 0; i < n; ++i)
    {
        C3 ri = c3(r[3 * i], r[3 * i + 1], r[3 * i + 2]), ni = c3(nv[3 * i], nv[3 * i + 1], nv[3 * i + 2]);
        int k = g.key(ri.x, ri.y, ri.z);
        int iz = k / (g.nx * g.ny), iy = (k / g.nx) % g.ny, ix = k % g.nx;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    int zz = iz + dz, yy = iy + dy, xx = ix + dx;
                    if (zz < 0 || yy < 0 || xx < 0 || zz >= g.nz || yy >= g.ny || xx >= g.nx) continue;
                    for (int j : g.bins[(size_t)(zz * g.ny + yy) * g.nx + xx])
                    {
                        if (j <= i) continue;
                        if (seg_dist(ri, ni, l[i] / 2, c3(r[3 * j], r[3 * j + 1], r[3 * j + 2]),
                                     c3(nv[3 * j], nv[3 * j + 1], nv[3 * j + 2]), l[j] / 2) < dist)
                            ++cnt;
                    }
                }
    }
    return cnt;
}
